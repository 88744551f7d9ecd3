// host_h5_write.cpp -- see host_h5_write.h.  The file is assembled in memory
// (members before the structures that point at them) and written once.
#include "host_h5_write.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <stdexcept>

namespace h5w {
namespace {

constexpr int kLeafK = 4;          // symbol table node: up to 2K entries
constexpr int kInternalK = 16;     // group B-tree node: up to 2K children
constexpr uint64_t kUndef = ~0ULL;
constexpr size_t kEntry = 40;      // symbol table entry with 8-byte offsets
constexpr uint64_t kHeapFreeNull = 1;   // "no next free block" in a local heap

size_t pad8(size_t n) { return (n + 7) & ~static_cast<size_t>(7); }

class Buf {
 public:
  uint64_t alloc(size_t n) {
    const size_t at = pad8(b_.size());
    b_.resize(at + n, 0);
    return at;
  }
  void put(uint64_t at, const void *p, size_t n) { std::memcpy(b_.data() + at, p, n); }
  template <typename T>
  void le(uint64_t at, T v) {
    for (size_t i = 0; i < sizeof(T); ++i) b_[at + i] = static_cast<uint8_t>(static_cast<uint64_t>(v) >> (8 * i));
  }
  size_t size() const { return b_.size(); }
  const std::vector<uint8_t> &bytes() const { return b_; }

 private:
  std::vector<uint8_t> b_;
};

std::vector<uint8_t> datatype(Type t) {
  std::vector<uint8_t> d;
  auto u32 = [&](uint32_t v) { for (int i = 0; i < 4; ++i) d.push_back(static_cast<uint8_t>(v >> (8 * i))); };
  auto u16 = [&](uint16_t v) { d.push_back(static_cast<uint8_t>(v)); d.push_back(static_cast<uint8_t>(v >> 8)); };
  if (t == Type::F64) {
    d = {0x11, 0x20, 0x3f, 0x00};   // version 1 floating point; IEEE, sign at bit 63
    u32(8);
    u16(0);
    u16(64);
    d.push_back(52);               // exponent location, size
    d.push_back(11);
    d.push_back(0);                // mantissa location, size
    d.push_back(52);
    u32(1023);
    return d;
  }
  const uint32_t size = t == Type::U8 ? 1 : t == Type::I32 ? 4 : 8;
  d = {0x10, static_cast<uint8_t>(t == Type::I32 ? 0x08 : 0x00), 0x00, 0x00};   // version 1 fixed point
  u32(size);
  u16(0);
  u16(static_cast<uint16_t>(8 * size));
  return d;
}

std::vector<uint8_t> dataspace(bool scalar, uint64_t n) {
  std::vector<uint8_t> d = {1, static_cast<uint8_t>(scalar ? 0 : 1), static_cast<uint8_t>(scalar ? 0 : 1),
                            0, 0, 0, 0, 0};
  if (!scalar)
    for (int rep = 0; rep < 2; ++rep)   // size, then maximum size
      for (int i = 0; i < 8; ++i) d.push_back(static_cast<uint8_t>(n >> (8 * i)));
  return d;
}

struct Msg {
  uint16_t type;
  uint8_t flags;
  std::vector<uint8_t> body;
};

Msg attr_msg(const Attr &a) {
  const std::vector<uint8_t> dt = datatype(a.type), ds = dataspace(a.scalar, a.count);
  const size_t nlen = a.name.size() + 1;
  Msg m{0x000C, 0, {}};
  std::vector<uint8_t> &b = m.body;
  b.assign(8 + pad8(nlen) + pad8(dt.size()) + pad8(ds.size()) + a.data.size(), 0);
  b[0] = 1;
  b[2] = static_cast<uint8_t>(nlen);
  b[3] = static_cast<uint8_t>(nlen >> 8);
  b[4] = static_cast<uint8_t>(dt.size());
  b[6] = static_cast<uint8_t>(ds.size());
  size_t o = 8;
  std::memcpy(b.data() + o, a.name.c_str(), nlen);
  o += pad8(nlen);
  std::memcpy(b.data() + o, dt.data(), dt.size());
  o += pad8(dt.size());
  std::memcpy(b.data() + o, ds.data(), ds.size());
  o += pad8(ds.size());
  if (!a.data.empty()) std::memcpy(b.data() + o, a.data.data(), a.data.size());
  return m;
}

// A version-1 object header holding `msgs`; returns its address.
uint64_t object_header(Buf &f, const std::vector<Msg> &msgs) {
  size_t body = 0;
  for (const Msg &m : msgs) body += 8 + pad8(m.body.size());
  const uint64_t at = f.alloc(16 + body);
  f.le<uint8_t>(at, 1);
  f.le<uint16_t>(at + 2, static_cast<uint16_t>(msgs.size()));
  f.le<uint32_t>(at + 4, 1);
  f.le<uint32_t>(at + 8, static_cast<uint32_t>(body));
  uint64_t p = at + 16;
  for (const Msg &m : msgs) {
    f.le<uint16_t>(p, m.type);
    f.le<uint16_t>(p + 2, static_cast<uint16_t>(pad8(m.body.size())));
    f.le<uint8_t>(p + 4, m.flags);
    if (!m.body.empty()) f.put(p + 8, m.body.data(), m.body.size());
    p += 8 + pad8(m.body.size());
  }
  return at;
}

struct GroupAddr {
  uint64_t header, btree, heap;
};

uint64_t write_dataset(Buf &f, const Dataset &d) {
  const uint64_t bytes = d.count * 8;
  const uint64_t data = f.alloc(bytes);
  if (bytes) f.put(data, d.data, bytes);
  std::vector<Msg> msgs;
  msgs.push_back(Msg{0x0001, 0, dataspace(false, d.count)});
  msgs.push_back(Msg{0x0003, 1, datatype(Type::U64)});
  msgs.push_back(Msg{0x0005, 1, {2, 2, 2, 1, 0, 0, 0, 0}});   // fill value v2: late alloc, default value
  Msg layout{0x0008, 0, std::vector<uint8_t>(18, 0)};
  layout.body[0] = 3;   // version 3, contiguous
  layout.body[1] = 1;
  for (int i = 0; i < 8; ++i) {
    layout.body[2 + i] = static_cast<uint8_t>(data >> (8 * i));
    layout.body[10 + i] = static_cast<uint8_t>(bytes >> (8 * i));
  }
  msgs.push_back(layout);
  for (const Attr &a : d.attrs) msgs.push_back(attr_msg(a));
  return object_header(f, msgs);
}

struct Member {
  std::string name;
  uint64_t header = 0, btree = 0, heap = 0;
  bool group = false;
  uint64_t name_off = 0;
};

GroupAddr write_group(Buf &f, const Group &g) {
  std::vector<Member> mem;
  for (const Group &c : g.groups) {
    const GroupAddr a = write_group(f, c);
    mem.push_back(Member{c.name, a.header, a.btree, a.heap, true});
  }
  for (const Dataset &d : g.datasets) mem.push_back(Member{d.name, write_dataset(f, d), 0, 0, false});
  std::sort(mem.begin(), mem.end(), [](const Member &a, const Member &b) { return a.name < b.name; });
  for (size_t i = 1; i < mem.size(); ++i)
    if (mem[i].name == mem[i - 1].name) throw std::runtime_error("duplicate HDF5 member " + mem[i].name);

  // local heap: "" at 0, the names, then one free block
  size_t seg = 8;
  for (Member &m : mem) {
    m.name_off = seg;
    seg += pad8(m.name.size() + 1);
  }
  const size_t free_at = seg;
  seg += 16;
  const uint64_t heap = f.alloc(32 + seg);
  f.put(heap, "HEAP", 4);
  f.le<uint64_t>(heap + 8, seg);
  f.le<uint64_t>(heap + 16, free_at);
  f.le<uint64_t>(heap + 24, heap + 32);
  for (const Member &m : mem) f.put(heap + 32 + m.name_off, m.name.c_str(), m.name.size() + 1);
  f.le<uint64_t>(heap + 32 + free_at, kHeapFreeNull);
  f.le<uint64_t>(heap + 32 + free_at + 8, 16);

  // symbol table nodes of up to 2 * kLeafK entries, name order
  struct Child {
    uint64_t addr, left_key, right_key;   // keys: heap offsets of names
  };
  std::vector<Child> level;
  const size_t per_node = 2 * kLeafK;
  for (size_t i = 0; i < mem.size(); i += per_node) {
    const size_t n = std::min(per_node, mem.size() - i);
    const uint64_t at = f.alloc(8 + per_node * kEntry);
    f.put(at, "SNOD", 4);
    f.le<uint8_t>(at + 4, 1);
    f.le<uint16_t>(at + 6, static_cast<uint16_t>(n));
    for (size_t j = 0; j < n; ++j) {
      const Member &m = mem[i + j];
      const uint64_t e = at + 8 + j * kEntry;
      f.le<uint64_t>(e, m.name_off);
      f.le<uint64_t>(e + 8, m.header);
      if (m.group) {
        f.le<uint32_t>(e + 16, 1);   // cached symbol table
        f.le<uint64_t>(e + 24, m.btree);
        f.le<uint64_t>(e + 32, m.heap);
      }
    }
    level.push_back(Child{at, level.empty() ? 0 : level.back().right_key, mem[i + n - 1].name_off});
  }

  // B-tree levels of up to 2 * kInternalK children until one root remains
  const size_t fan = 2 * kInternalK;
  const size_t node_bytes = 24 + (2 * kInternalK + 1) * 8 + 2 * kInternalK * 8;
  int depth = 0;
  do {
    std::vector<Child> up;
    std::vector<uint64_t> addrs;
    for (size_t i = 0; i < level.size() || (i == 0 && level.empty()); i += fan) {
      const size_t n = level.empty() ? 0 : std::min(fan, level.size() - i);
      const uint64_t at = f.alloc(node_bytes);
      f.put(at, "TREE", 4);
      f.le<uint8_t>(at + 4, 0);   // group node
      f.le<uint8_t>(at + 5, static_cast<uint8_t>(depth));
      f.le<uint16_t>(at + 6, static_cast<uint16_t>(n));
      f.le<uint64_t>(at + 8, kUndef);
      f.le<uint64_t>(at + 16, kUndef);
      uint64_t p = at + 24;
      f.le<uint64_t>(p, n ? level[i].left_key : 0);
      p += 8;
      for (size_t j = 0; j < n; ++j) {
        f.le<uint64_t>(p, level[i + j].addr);
        f.le<uint64_t>(p + 8, level[i + j].right_key);
        p += 16;
      }
      addrs.push_back(at);
      up.push_back(Child{at, n ? level[i].left_key : 0, n ? level[i + n - 1].right_key : 0});
      if (level.empty()) break;
    }
    for (size_t j = 0; j < addrs.size(); ++j) {   // siblings on this level
      if (j > 0) f.le<uint64_t>(addrs[j] + 8, addrs[j - 1]);
      if (j + 1 < addrs.size()) f.le<uint64_t>(addrs[j] + 16, addrs[j + 1]);
    }
    level.swap(up);
    ++depth;
  } while (level.size() > 1);

  std::vector<Msg> msgs;
  Msg symtab{0x0011, 0, std::vector<uint8_t>(16, 0)};
  for (int i = 0; i < 8; ++i) {
    symtab.body[i] = static_cast<uint8_t>(level[0].addr >> (8 * i));
    symtab.body[8 + i] = static_cast<uint8_t>(heap >> (8 * i));
  }
  msgs.push_back(symtab);
  for (const Attr &a : g.attrs) msgs.push_back(attr_msg(a));
  return GroupAddr{object_header(f, msgs), level[0].addr, heap};
}

}  // namespace

Attr Attr::u8(const std::string &n, uint8_t v) {
  Attr a;
  a.name = n;
  a.type = Type::U8;
  a.data = {v};
  return a;
}

Attr Attr::u64(const std::string &n, uint64_t v) {
  Attr a;
  a.name = n;
  a.type = Type::U64;
  a.data.resize(8);
  for (int i = 0; i < 8; ++i) a.data[i] = static_cast<uint8_t>(v >> (8 * i));
  return a;
}

Attr Attr::i32(const std::string &n, int32_t v) {
  Attr a = i32_vec(n, {v});
  a.scalar = true;
  return a;
}

Attr Attr::i32_vec(const std::string &n, const std::vector<int32_t> &v) {
  Attr a;
  a.name = n;
  a.type = Type::I32;
  a.scalar = false;
  a.count = v.size();
  a.data.resize(4 * v.size());
  std::memcpy(a.data.data(), v.data(), v.size() * sizeof(int32_t));
  return a;
}

Attr Attr::f64_vec(const std::string &n, const std::vector<double> &v) {
  Attr a;
  a.name = n;
  a.type = Type::F64;
  a.scalar = false;
  a.count = v.size();
  a.data.resize(8 * v.size());
  std::memcpy(a.data.data(), v.data(), a.data.size());
  return a;
}

void write_file(const std::string &path, const Group &root) {
  Buf f;
  const uint64_t sb = f.alloc(96);
  const GroupAddr r = write_group(f, root);
  static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  f.put(sb, sig, 8);
  f.le<uint8_t>(sb + 13, 8);              // size of offsets
  f.le<uint8_t>(sb + 14, 8);              // size of lengths
  f.le<uint16_t>(sb + 16, kLeafK);
  f.le<uint16_t>(sb + 18, kInternalK);
  f.le<uint64_t>(sb + 24, 0);             // base address
  f.le<uint64_t>(sb + 32, kUndef);        // free-space info
  f.le<uint64_t>(sb + 40, f.size());      // end of file
  f.le<uint64_t>(sb + 48, kUndef);        // driver information
  f.le<uint64_t>(sb + 56, 0);             // root entry: name offset
  f.le<uint64_t>(sb + 64, r.header);
  f.le<uint32_t>(sb + 72, 1);
  f.le<uint64_t>(sb + 80, r.btree);
  f.le<uint64_t>(sb + 88, r.heap);
  FILE *fp = std::fopen(path.c_str(), "wb");
  if (!fp) throw std::runtime_error("Could not create " + path);
  const size_t n = std::fwrite(f.bytes().data(), 1, f.size(), fp);
  const int closed = std::fclose(fp);
  if (n != f.size() || closed != 0) throw std::runtime_error("Could not write " + path);
}

}  // namespace h5w
