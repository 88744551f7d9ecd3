// host_h5_write.h -- writes the subset of HDF5 that pp-sketchlib's sketch
// databases use, so constructDatabase needs no libhdf5.
//
// The structures are the ones libhdf5 writes by default and the reference's
// databases hold (src/database/database.cpp:40-258 through HighFive):
// superblock version 0 (group leaf node K 4, internal node K 16), version-1
// object headers, groups as symbol tables (version-1 B-tree, symbol table
// nodes, local heap ending in a free block), version-1 attribute messages,
// contiguous datasets with version-2 fill value and version-3 layout
// messages.  Scalars are scalar dataspaces, vectors one-dimensional ones with
// their maximum dimension equal to the size, all little endian.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace h5w {

enum class Type { U8, I32, U64, F64 };

struct Attr {
  std::string name;
  Type type = Type::U64;
  bool scalar = true;             // false: one-dimensional of `count` elements
  uint64_t count = 1;
  std::vector<uint8_t> data;      // count elements, little endian

  static Attr u8(const std::string &n, uint8_t v);
  static Attr u64(const std::string &n, uint64_t v);
  static Attr i32(const std::string &n, int32_t v);
  static Attr i32_vec(const std::string &n, const std::vector<int32_t> &v);
  static Attr f64_vec(const std::string &n, const std::vector<double> &v);
};

struct Dataset {
  std::string name;
  const uint64_t *data = nullptr;  // `count` little-endian uint64 values
  uint64_t count = 0;
  std::vector<Attr> attrs;
};

struct Group {
  std::string name;
  std::vector<Attr> attrs;
  std::vector<Group> groups;
  std::vector<Dataset> datasets;
};

// Writes `root` (its name is ignored) as a new file at `path`, replacing any
// file there.  Member names within a group must be unique.  Throws
// std::runtime_error on I/O errors.
void write_file(const std::string &path, const Group &root);

}  // namespace h5w
