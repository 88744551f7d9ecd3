// host_h5.h -- a read-only reader for the subset of HDF5 that pp-sketchlib's
// sketch databases use, so the drop-in module needs no libhdf5.
//
// The reference writes its databases through HighFive with libhdf5's default
// (earliest) file format (src/database/database.cpp:23-258): superblock
// version 0/1, version-1 object headers, groups as symbol tables (v1 B-tree +
// local heap), contiguous or compact datasets of fixed-size integers and
// floats, attributes as header messages, and variable-length strings in global
// heap collections.  That is what this reader implements; anything else
// (chunked/filtered data, version-2 object headers, dense link storage) is
// reported as an error naming the unsupported feature.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace h5 {

struct Error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// A fixed-size element type.
struct DType {
  int cls = -1;        // 0 integer, 1 float, 3 fixed string, 9 variable length
  int size = 0;        // bytes per element
  bool is_signed = false;
  bool vlen_string = false;
};

struct Space {
  std::vector<uint64_t> dims;  // empty for a scalar
  uint64_t count() const;
};

// A decoded object: header messages we care about.
struct Object {
  uint64_t addr = 0;
  bool is_group = false;
  uint64_t btree = 0, heap = 0;     // group: symbol table
  DType dtype;                      // dataset
  Space space;
  int layout = -1;                  // 0 compact, 1 contiguous
  uint64_t data_addr = 0, data_size = 0;
  std::vector<uint8_t> compact;
  struct Attr {
    std::string name;
    DType dtype;
    Space space;
    std::vector<uint8_t> data;
  };
  std::vector<Attr> attrs;
};

class File {
 public:
  explicit File(const std::string &path);
  ~File();
  File(const File &) = delete;
  File &operator=(const File &) = delete;

  // Object at an absolute path ("/", "/sketches/name/15").  Throws if absent.
  Object open(const std::string &path) const;
  bool exists(const std::string &path) const;
  // Names of a group's members, in the group's (name-sorted) B-tree order.
  std::vector<std::string> list(const Object &group) const;
  // A group's members by name (one walk of its B-tree), and the object at a
  // member's header address: opening many members of one large group costs
  // one walk instead of one per member.
  std::unordered_map<std::string, uint64_t> members(const Object &group) const;
  Object object_at(uint64_t addr) const { return decode(addr); }

  // Attribute / dataset values converted to the requested element type.
  static bool has_attr(const Object &o, const std::string &name);
  std::vector<int64_t> attr_ints(const Object &o, const std::string &name) const;
  std::vector<double> attr_doubles(const Object &o, const std::string &name) const;
  std::vector<int64_t> read_ints(const Object &ds) const;
  std::vector<double> read_doubles(const Object &ds) const;
  std::vector<std::string> read_strings(const Object &ds) const;
  // Raw little-endian 8-byte words of an unsigned 64-bit dataset, copied to dst
  // (which holds at least count() words).
  void read_u64(const Object &ds, uint64_t *dst) const;

  const std::string &path() const { return path_; }

 private:
  Object decode(uint64_t addr) const;
  const uint8_t *at(uint64_t off, uint64_t len) const;
  uint64_t off(const uint8_t *p) const;  // reads an offset-sized field
  uint64_t len(const uint8_t *p) const;  // reads a length-sized field
  uint64_t lookup(const Object &group, const std::string &name, bool *found) const;
  void walk_btree(uint64_t addr, const uint8_t *heap, uint64_t heap_size,
                  std::vector<std::pair<std::string, uint64_t>> &out, int depth) const;
  std::vector<uint8_t> element_bytes(const Object &ds) const;
  std::string vlen_string(const uint8_t *p) const;

  std::string path_;
  const uint8_t *data_ = nullptr;
  size_t size_ = 0;
  int fd_ = -1;
  int off_size_ = 8, len_size_ = 8;
  uint64_t base_ = 0, root_ = 0;
};

}  // namespace h5
