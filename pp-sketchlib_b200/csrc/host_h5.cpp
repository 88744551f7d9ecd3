// host_h5.cpp -- see host_h5.h.  Field layouts follow the published HDF5
// file-format specification (superblock v0/v1, object header v1, symbol
// table / v1 B-tree / local heap, global heap collections).
#include "host_h5.h"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstring>
#include <functional>
#include <sstream>

namespace h5 {
namespace {

constexpr uint8_t kSignature[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

uint64_t rd(const uint8_t *p, int n) {
  uint64_t v = 0;
  for (int i = n - 1; i >= 0; --i) v = (v << 8) | p[i];
  return v;
}

size_t pad8(size_t n) { return (n + 7) & ~static_cast<size_t>(7); }

}  // namespace

uint64_t Space::count() const {
  uint64_t c = 1;
  for (uint64_t d : dims) c *= d;
  return c;
}

File::File(const std::string &path) : path_(path) {
  fd_ = ::open(path.c_str(), O_RDONLY);
  if (fd_ < 0) throw Error("Unable to open file " + path);
  struct stat st {};
  if (fstat(fd_, &st) != 0 || st.st_size < 64) {
    ::close(fd_);
    throw Error("Not an HDF5 file: " + path);
  }
  size_ = static_cast<size_t>(st.st_size);
  void *m = mmap(nullptr, size_, PROT_READ, MAP_PRIVATE, fd_, 0);
  if (m == MAP_FAILED) {
    ::close(fd_);
    throw Error("Unable to map file " + path);
  }
  data_ = static_cast<const uint8_t *>(m);
  // the superblock sits at 0, 512, 1024, 2048, ...
  size_t sb = std::string::npos;
  for (size_t o = 0; o + 8 <= size_; o = o ? o * 2 : 512) {
    if (std::memcmp(data_ + o, kSignature, 8) == 0) {
      sb = o;
      break;
    }
  }
  if (sb == std::string::npos) throw Error("Not an HDF5 file (no signature): " + path);
  const uint8_t *p = data_ + sb;
  const int version = p[8];
  if (version > 1)
    throw Error("HDF5 superblock version " + std::to_string(version) +
                " is not supported (the reference writes version 0)");
  off_size_ = p[13];
  len_size_ = p[14];
  if ((off_size_ != 4 && off_size_ != 8) || (len_size_ != 4 && len_size_ != 8))
    throw Error("unsupported HDF5 offset/length sizes");
  size_t q = sb + 24 + (version == 1 ? 4 : 0);
  base_ = rd(data_ + q, off_size_);
  q += 4 * off_size_;  // base, free-space, end of file, driver info
  // root group symbol table entry: link name offset, object header address
  root_ = rd(data_ + q + off_size_, off_size_);
}

File::~File() {
  if (data_) munmap(const_cast<uint8_t *>(data_), size_);
  if (fd_ >= 0) ::close(fd_);
}

const uint8_t *File::at(uint64_t off, uint64_t len) const {
  const uint64_t a = base_ + off;
  if (a > size_ || len > size_ - a) throw Error("HDF5 structure points outside " + path_);
  return data_ + a;
}

uint64_t File::off(const uint8_t *p) const { return rd(p, off_size_); }
uint64_t File::len(const uint8_t *p) const { return rd(p, len_size_); }

static DType parse_dtype(const uint8_t *p, size_t n) {
  if (n < 8) throw Error("truncated HDF5 datatype");
  DType t;
  t.cls = p[0] & 0x0f;
  const uint32_t bits = static_cast<uint32_t>(rd(p + 1, 3));
  t.size = static_cast<int>(rd(p + 4, 4));
  if (t.cls == 0) {
    if (bits & 1u) throw Error("big-endian HDF5 integers are not supported");
    t.is_signed = (bits & 8u) != 0;
  } else if (t.cls == 1) {
    if (bits & 1u) throw Error("big-endian HDF5 floats are not supported");
  } else if (t.cls == 9) {
    t.vlen_string = (bits & 0x0f) == 1;
  }
  return t;
}

static Space parse_space(const uint8_t *p, size_t n, int len_size) {
  if (n < 4) throw Error("truncated HDF5 dataspace");
  Space s;
  const int version = p[0], rank = p[1];
  size_t q;
  if (version == 1) {
    q = 8;
  } else if (version == 2) {
    q = 4;
    if (p[3] == 2) return s;  // null dataspace: treat as scalar
  } else {
    throw Error("unsupported HDF5 dataspace version");
  }
  for (int r = 0; r < rank; ++r) {
    if (q + len_size > n) throw Error("truncated HDF5 dataspace");
    s.dims.push_back(rd(p + q, len_size));
    q += len_size;
  }
  return s;
}

Object File::decode(uint64_t addr) const {
  Object o;
  o.addr = addr;
  const uint8_t *h = at(addr, 16);
  if (h[0] != 1) {
    if (std::memcmp(h, "OHDR", 4) == 0)
      throw Error("version-2 HDF5 object headers are not supported (file written with a newer "
                  "format than the reference uses)");
    throw Error("bad HDF5 object header");
  }
  const uint32_t nmsg = static_cast<uint32_t>(rd(h + 2, 2));
  std::vector<std::pair<uint64_t, uint64_t>> blocks{{addr + 16, rd(h + 8, 4)}};
  uint32_t seen = 0;
  for (size_t bi = 0; bi < blocks.size() && seen < nmsg; ++bi) {
    uint64_t pos = blocks[bi].first;
    const uint64_t end = pos + blocks[bi].second;
    while (pos + 8 <= end && seen < nmsg) {
      const uint8_t *m = at(pos, 8);
      const int type = static_cast<int>(rd(m, 2));
      const size_t msz = static_cast<size_t>(rd(m + 2, 2));
      const int flags = m[4];
      const uint8_t *d = at(pos + 8, msz);
      pos += 8 + msz;
      ++seen;
      if ((flags & 2) && (type == 1 || type == 3))
        throw Error("shared HDF5 header messages are not supported");
      switch (type) {
        case 0x0001: o.space = parse_space(d, msz, len_size_); break;
        case 0x0003: o.dtype = parse_dtype(d, msz); break;
        case 0x0008: {
          const int version = d[0];
          if (version >= 3) {
            o.layout = d[1];
            if (o.layout == 0) {
              const size_t n = static_cast<size_t>(rd(d + 2, 2));
              o.compact.assign(d + 4, d + 4 + n);
            } else if (o.layout == 1) {
              o.data_addr = off(d + 2);
              o.data_size = len(d + 2 + off_size_);
            } else {
              throw Error("chunked or virtual HDF5 datasets are not supported");
            }
          } else {
            const int rank = d[1];
            o.layout = d[2];
            if (o.layout == 1) {
              o.data_addr = off(d + 8);
            } else if (o.layout == 0) {
              const size_t q = 8 + 4 * static_cast<size_t>(rank);
              const size_t n = static_cast<size_t>(rd(d + q, 4));
              o.compact.assign(d + q + 4, d + q + 4 + n);
            } else {
              throw Error("chunked HDF5 datasets are not supported");
            }
          }
          break;
        }
        case 0x000C: {
          Object::Attr a;
          const int version = d[0];
          const size_t nlen = static_cast<size_t>(rd(d + 2, 2));
          const size_t tlen = static_cast<size_t>(rd(d + 4, 2));
          const size_t slen = static_cast<size_t>(rd(d + 6, 2));
          size_t q = version == 3 ? 9 : 8;
          auto adv = [&](size_t n) { return version == 1 ? pad8(n) : n; };
          a.name.assign(reinterpret_cast<const char *>(d + q), nlen ? strnlen(reinterpret_cast<const char *>(d + q), nlen) : 0);
          q += adv(nlen);
          a.dtype = parse_dtype(d + q, tlen);
          q += adv(tlen);
          a.space = parse_space(d + q, slen, len_size_);
          q += adv(slen);
          const size_t bytes = static_cast<size_t>(a.space.count()) * a.dtype.size;
          if (q + bytes > msz) throw Error("truncated HDF5 attribute " + a.name);
          a.data.assign(d + q, d + q + bytes);
          o.attrs.push_back(std::move(a));
          break;
        }
        case 0x0010: blocks.emplace_back(off(d), len(d + off_size_)); break;
        case 0x0011:
          o.is_group = true;
          o.btree = off(d);
          o.heap = off(d + off_size_);
          break;
        case 0x0002:  // link info: a new-style group
        case 0x0006:  // link
          throw Error("new-style HDF5 groups (link messages) are not supported");
        default: break;
      }
    }
  }
  return o;
}

void File::walk_btree(uint64_t addr, const uint8_t *heap, uint64_t heap_size,
                      std::vector<std::pair<std::string, uint64_t>> &out, int depth) const {
  if (depth > 64) throw Error("HDF5 B-tree too deep");
  const uint8_t *n = at(addr, 8 + 2 * off_size_);
  if (std::memcmp(n, "TREE", 4) != 0 || n[4] != 0) throw Error("bad HDF5 group B-tree node");
  const int level = n[5];
  const int used = static_cast<int>(rd(n + 6, 2));
  const uint64_t first = addr + 8 + 2 * off_size_;
  const uint64_t stride = len_size_ + off_size_;
  for (int i = 0; i < used; ++i) {
    const uint64_t child = off(at(first + i * stride + len_size_, off_size_));
    if (level > 0) {
      walk_btree(child, heap, heap_size, out, depth + 1);
      continue;
    }
    const uint8_t *s = at(child, 8);
    if (std::memcmp(s, "SNOD", 4) != 0) throw Error("bad HDF5 symbol table node");
    const int nsym = static_cast<int>(rd(s + 6, 2));
    const uint64_t ste = 2 * off_size_ + 24;
    for (int e = 0; e < nsym; ++e) {
      const uint8_t *en = at(child + 8 + e * ste, ste);
      const uint64_t name_off = off(en);
      const uint64_t oh = off(en + off_size_);
      if (name_off >= heap_size) throw Error("bad HDF5 link name offset");
      const char *nm = reinterpret_cast<const char *>(heap + name_off);
      out.emplace_back(std::string(nm, strnlen(nm, heap_size - name_off)), oh);
    }
  }
}

std::vector<std::string> File::list(const Object &group) const {
  if (!group.is_group) throw Error("not an HDF5 group");
  const uint8_t *h = at(group.heap, 8 + 2 * len_size_ + off_size_);
  if (std::memcmp(h, "HEAP", 4) != 0) throw Error("bad HDF5 local heap");
  const uint64_t heap_size = len(h + 8);
  const uint64_t heap_addr = off(h + 8 + 2 * len_size_);
  const uint8_t *heap = at(heap_addr, heap_size);
  std::vector<std::pair<std::string, uint64_t>> entries;
  walk_btree(group.btree, heap, heap_size, entries, 0);
  std::vector<std::string> names;
  names.reserve(entries.size());
  for (auto &e : entries) names.push_back(e.first);
  return names;
}

std::unordered_map<std::string, uint64_t> File::members(const Object &group) const {
  if (!group.is_group) throw Error("not an HDF5 group");
  const uint8_t *h = at(group.heap, 8 + 2 * len_size_ + off_size_);
  if (std::memcmp(h, "HEAP", 4) != 0) throw Error("bad HDF5 local heap");
  const uint64_t heap_size = len(h + 8);
  const uint8_t *heap = at(off(h + 8 + 2 * len_size_), heap_size);
  std::vector<std::pair<std::string, uint64_t>> entries;
  walk_btree(group.btree, heap, heap_size, entries, 0);
  std::unordered_map<std::string, uint64_t> out;
  out.reserve(entries.size());
  for (auto &e : entries) out.emplace(std::move(e.first), e.second);
  return out;
}

uint64_t File::lookup(const Object &group, const std::string &name, bool *found) const {
  *found = false;
  if (!group.is_group) return 0;
  const uint8_t *h = at(group.heap, 8 + 2 * len_size_ + off_size_);
  if (std::memcmp(h, "HEAP", 4) != 0) throw Error("bad HDF5 local heap");
  const uint64_t heap_size = len(h + 8);
  const uint8_t *heap = at(off(h + 8 + 2 * len_size_), heap_size);
  std::vector<std::pair<std::string, uint64_t>> entries;
  walk_btree(group.btree, heap, heap_size, entries, 0);
  for (auto &e : entries) {
    if (e.first == name) {
      *found = true;
      return e.second;
    }
  }
  return 0;
}

Object File::open(const std::string &path) const {
  Object cur = decode(root_);
  std::stringstream ss(path);
  std::string part;
  std::string walked;
  while (std::getline(ss, part, '/')) {
    if (part.empty()) continue;
    walked += "/" + part;
    bool found = false;
    const uint64_t a = lookup(cur, part, &found);
    if (!found) throw Error("Object " + walked + " does not exist in " + path_);
    cur = decode(a);
  }
  return cur;
}

bool File::exists(const std::string &path) const {
  try {
    open(path);
    return true;
  } catch (const Error &) {
    return false;
  }
}

bool File::has_attr(const Object &o, const std::string &name) {
  for (auto &a : o.attrs)
    if (a.name == name) return true;
  return false;
}

template <typename T>
static std::vector<T> convert(const DType &t, const uint8_t *p, uint64_t n, const std::string &what) {
  std::vector<T> out(n);
  for (uint64_t i = 0; i < n; ++i) {
    const uint8_t *e = p + i * t.size;
    if (t.cls == 0) {
      uint64_t u = rd(e, t.size);
      if (t.is_signed && t.size < 8 && (u >> (8 * t.size - 1)) & 1u) u |= ~0ull << (8 * t.size);
      out[i] = t.is_signed ? static_cast<T>(static_cast<int64_t>(u)) : static_cast<T>(u);
    } else if (t.cls == 1 && t.size == 8) {
      double d;
      std::memcpy(&d, e, 8);
      out[i] = static_cast<T>(d);
    } else if (t.cls == 1 && t.size == 4) {
      float f;
      std::memcpy(&f, e, 4);
      out[i] = static_cast<T>(f);
    } else {
      throw Error("unsupported HDF5 element type for " + what);
    }
  }
  return out;
}

std::vector<int64_t> File::attr_ints(const Object &o, const std::string &name) const {
  for (auto &a : o.attrs)
    if (a.name == name) return convert<int64_t>(a.dtype, a.data.data(), a.space.count(), name);
  throw Error("Attribute " + name + " not found");
}

std::vector<double> File::attr_doubles(const Object &o, const std::string &name) const {
  for (auto &a : o.attrs)
    if (a.name == name) return convert<double>(a.dtype, a.data.data(), a.space.count(), name);
  throw Error("Attribute " + name + " not found");
}

std::vector<uint8_t> File::element_bytes(const Object &ds) const {
  const uint64_t bytes = ds.space.count() * static_cast<uint64_t>(ds.dtype.size);
  if (ds.layout == 0) {
    if (ds.compact.size() < bytes) throw Error("truncated compact HDF5 dataset");
    return std::vector<uint8_t>(ds.compact.begin(), ds.compact.begin() + bytes);
  }
  if (ds.layout != 1) throw Error("not an HDF5 dataset");
  if (ds.data_addr == ~0ull || bytes == 0) return std::vector<uint8_t>(bytes, 0);  // never written
  const uint8_t *p = at(ds.data_addr, bytes);
  return std::vector<uint8_t>(p, p + bytes);
}

std::vector<int64_t> File::read_ints(const Object &ds) const {
  auto b = element_bytes(ds);
  return convert<int64_t>(ds.dtype, b.data(), ds.space.count(), "dataset");
}

std::vector<double> File::read_doubles(const Object &ds) const {
  auto b = element_bytes(ds);
  return convert<double>(ds.dtype, b.data(), ds.space.count(), "dataset");
}

void File::read_u64(const Object &ds, uint64_t *dst) const {
  if (ds.dtype.cls != 0 || ds.dtype.size != 8) throw Error("sketch dataset is not 64-bit integers");
  const uint64_t n = ds.space.count();
  if (ds.layout == 1 && ds.data_addr != ~0ull) {
    std::memcpy(dst, at(ds.data_addr, n * 8), n * 8);
  } else {
    auto b = element_bytes(ds);
    std::memcpy(dst, b.data(), n * 8);
  }
}

// A variable-length string element: length, global heap collection, index.
std::string File::vlen_string(const uint8_t *p) const {
  const uint64_t n = rd(p, 4);
  const uint64_t coll = off(p + 4);
  const uint64_t idx = rd(p + 4 + off_size_, 4);
  if (n == 0) return std::string();
  const uint8_t *c = at(coll, 8 + len_size_);
  if (std::memcmp(c, "GCOL", 4) != 0) throw Error("bad HDF5 global heap collection");
  const uint64_t csize = len(c + 8);
  uint64_t pos = coll + 8 + len_size_;
  const uint64_t end = coll + csize;
  while (pos + 8 + len_size_ <= end) {
    const uint8_t *ob = at(pos, 8 + len_size_);
    const uint64_t oidx = rd(ob, 2);
    const uint64_t osz = len(ob + 8);
    if (oidx == 0) break;  // free space
    if (oidx == idx) {
      const uint8_t *s = at(pos + 8 + len_size_, osz);
      return std::string(reinterpret_cast<const char *>(s), std::min<uint64_t>(osz, n));
    }
    pos += 8 + len_size_ + pad8(osz);
  }
  throw Error("HDF5 global heap object not found");
}

std::vector<std::string> File::read_strings(const Object &ds) const {
  auto b = element_bytes(ds);
  const uint64_t n = ds.space.count();
  std::vector<std::string> out;
  out.reserve(n);
  for (uint64_t i = 0; i < n; ++i) {
    const uint8_t *e = b.data() + i * ds.dtype.size;
    if (ds.dtype.cls == 9) {
      out.push_back(vlen_string(e));
    } else if (ds.dtype.cls == 3) {
      const char *s = reinterpret_cast<const char *>(e);
      out.emplace_back(s, strnlen(s, ds.dtype.size));
    } else {
      throw Error("dataset is not a string array");
    }
  }
  return out;
}

}  // namespace h5
