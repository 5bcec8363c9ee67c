// The HDF5 reader of h5.h, following the published HDF5 file-format specification (superblock,
// object headers and their messages, v1 B-trees, local heaps, symbol-table nodes, the filter
// pipeline). Every address is bounds-checked against the file; anything outside the subset
// raises std::runtime_error naming what it met.
#include "h5.h"

#include <zlib.h>

#include <algorithm>
#include <cstring>
#include <fstream>
#include <iterator>
#include <stdexcept>

namespace ptyb::h5 {
namespace {

[[noreturn]] void fail(const std::string& what) { throw std::runtime_error("HDF5: " + what); }

constexpr int kMaxDepth = 64;
constexpr uint64_t kMaxNodes = 1u << 22;       // B-tree nodes one read may visit
constexpr uint64_t kMaxBytes = 1ull << 42;     // the largest dataset read (4 TiB)
constexpr uint64_t kMaxWork = 1ull << 24;      // work units one public call may spend
// A dataset is at most what its file can hold: deflate expands at most ~1032:1.
constexpr uint64_t kMaxExpansion = 1100;

// Fails unless [o, o + k) lies within a field of n bytes.
inline void need(size_t o, size_t k, size_t n, const char* what) {
  if (o > n || k > n - o) fail(std::string("truncated ") + what);
}

uint64_t le(const uint8_t* p, int n) {
  uint64_t v = 0;
  for (int i = n - 1; i >= 0; --i) v = (v << 8) | p[i];
  return v;
}

bool undefined(uint64_t addr, int so) {
  return so >= 8 ? addr == ~0ull : addr == ((1ull << (8 * so)) - 1);
}

// Parses a datatype message at p (at most n bytes); *used receives its length.
Type parse_type(const uint8_t* p, size_t n, size_t* used, int depth = 0) {
  need(0, 8, n, "datatype");
  if (depth > 8) fail("datatype nested too deeply");
  Type t;
  const int cls = p[0] & 15, version = p[0] >> 4;
  const uint32_t bits = (uint32_t)le(p + 1, 3);
  t.size = (uint32_t)le(p + 4, 4);
  size_t o = 8;
  switch (cls) {
    case Type::kFixed:
      t.cls = Type::kFixed;
      t.big_endian = bits & 1;
      t.is_signed = (bits >> 3) & 1;
      need(o, 4, n, "fixed-point datatype");
      o += 4;
      break;
    case Type::kFloat:
      t.cls = Type::kFloat;
      t.big_endian = bits & 1;
      need(o, 12, n, "floating-point datatype");
      o += 12;
      break;
    case Type::kString:
      t.cls = Type::kString;
      break;
    case Type::kCompound: {
      t.cls = Type::kCompound;
      const int nmem = (int)(bits & 0xffff);
      for (int k = 0; k < nmem; ++k) {
        need(o, 1, n, "compound datatype");
        const char* name = reinterpret_cast<const char*>(p + o);
        const size_t len = strnlen(name, n - o);
        Type::Member m;
        m.name.assign(name, len);
        if (version < 3) {
          o += (len + 8) / 8 * 8;  // name with its terminator, padded to 8 bytes
          need(o, 4, n, "compound member");
          m.offset = (uint32_t)le(p + o, 4);
          o += 4;
          if (version == 1) o += 1 + 3 + 4 + 4 + 16;  // dimensionality, permutation, sizes
        } else {
          o += len + 1;
          int ob = 1;
          while (ob < 4 && (t.size >> (8 * ob))) ++ob;
          need(o, ob, n, "compound member");
          m.offset = (uint32_t)le(p + o, ob);
          o += ob;
        }
        need(o, 8, n, "compound member type");
        size_t u = 0;
        m.type = std::make_shared<Type>(parse_type(p + o, n - o, &u, depth + 1));
        o += u;
        t.members.push_back(m);
      }
      break;
    }
    case Type::kEnum: {
      t.cls = Type::kEnum;
      const int nmem = (int)(bits & 0xffff);
      size_t u = 0;
      need(o, 8, n, "enumeration base type");
      t.base = std::make_shared<Type>(parse_type(p + o, n - o, &u, depth + 1));
      o += u;
      for (int k = 0; k < nmem; ++k) {  // the names
        need(o, 1, n, "enumeration names");
        const size_t len = strnlen(reinterpret_cast<const char*>(p + o), n - o);
        o += version < 3 ? (len + 8) / 8 * 8 : len + 1;
      }
      o += (size_t)nmem * t.base->size;  // the values
      need(0, o, n, "enumeration values");
      break;
    }
    default:
      t.cls = Type::kOther;
      break;
  }
  *used = o;
  return t;
}

// Undoes HDF5's shuffle filter: byte b of element i was stored at b·n + i.
std::vector<uint8_t> unshuffle(const std::vector<uint8_t>& in, size_t es) {
  const size_t n = es > 1 ? in.size() / es : 0;
  if (n == 0) return in;
  std::vector<uint8_t> out(in.size());
  for (size_t b = 0; b < es; ++b)
    for (size_t i = 0; i < n; ++i) out[i * es + b] = in[b * n + i];
  std::copy(in.begin() + n * es, in.end(), out.begin() + n * es);
  return out;
}

std::vector<uint8_t> inflate_all(const std::vector<uint8_t>& in, size_t expect) {
  std::vector<uint8_t> out(expect);
  z_stream z = {};
  if (inflateInit(&z) != Z_OK) fail("zlib init");
  z.next_in = const_cast<Bytef*>(in.data());
  z.avail_in = (uInt)in.size();
  z.next_out = out.data();
  z.avail_out = (uInt)out.size();
  const int rc = inflate(&z, Z_FINISH);
  const size_t got = out.size() - z.avail_out;
  inflateEnd(&z);
  if (rc != Z_STREAM_END || got != expect) fail("a deflate chunk did not expand to its size");
  return out;
}

struct Filter {
  int id;
  int flags;
  std::vector<uint32_t> values;
};

std::vector<Filter> parse_filters(const uint8_t* p, size_t n) {
  std::vector<Filter> out;
  need(0, 2, n, "filter pipeline");
  const int version = p[0], nf = p[1];
  size_t o = version == 1 ? 8 : 2;
  for (int k = 0; k < nf; ++k) {
    need(o, 8, n, "filter description");
    Filter f;
    f.id = (int)le(p + o, 2);
    o += 2;
    size_t namelen = 0;
    if (version == 1 || f.id >= 256) {
      namelen = le(p + o, 2);
      o += 2;
    }
    need(o, 4, n, "filter description");
    f.flags = (int)le(p + o, 2);
    const int nv = (int)le(p + o + 2, 2);
    o += 4;
    o += version == 1 ? (namelen + 7) / 8 * 8 : namelen;
    need(o, 4 * (size_t)nv, n, "filter client data");
    for (int v = 0; v < nv; ++v, o += 4) f.values.push_back((uint32_t)le(p + o, 4));
    if (version == 1 && (nv & 1)) o += 4;
    out.push_back(f);
  }
  return out;
}

}  // namespace

File::File(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) fail("cannot open " + path);
  buf_.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  uint64_t sb = ~0ull;
  for (uint64_t at = 0; at + 64 <= buf_.size(); at = at ? at * 2 : 512)
    if (!memcmp(&buf_[at], sig, 8)) {
      sb = at;
      break;
    }
  if (sb == ~0ull) fail(path + " is not an HDF5 file");
  const uint8_t* p = &buf_[sb + 8];
  const size_t room = buf_.size() - (sb + 8);
  const int version = p[0];
  if (version <= 1) {
    so_ = p[5];
    sl_ = p[6];
  } else if (version == 2 || version == 3) {
    so_ = p[1];
    sl_ = p[2];
  } else {
    fail("superblock version " + std::to_string(version));
  }
  if ((so_ != 4 && so_ != 8) || (sl_ != 4 && sl_ != 8)) fail("unsupported offset size");
  if (version <= 1) {
    size_t o = version == 1 ? 20 : 16;
    need(o, 6 * (size_t)so_, room, "superblock");
    base_ = le(p + o, so_);
    o += 4 * (size_t)so_;  // base, free-space, end-of-file and driver addresses
    root_ = le(p + o + so_, so_);  // the root entry's object header address
  } else {
    need(4, 4 * (size_t)so_, room, "superblock");
    base_ = le(p + 4, so_);
    root_ = le(p + 4 + 3 * (size_t)so_, so_);
  }
}

const uint8_t* File::ptr(uint64_t addr, uint64_t n) const {
  const uint64_t at = base_ + addr;
  if (at < addr || at > buf_.size() || n > buf_.size() - at) fail("address out of the file");
  return buf_.data() + at;
}

uint64_t File::uint_at(uint64_t at, int n) const { return le(ptr(at, n), n); }

void File::spend(uint64_t units) const {
  work_ += units;
  if (work_ > kMaxWork) fail("the file's structure does not end (a cycle)");
}

void File::collect(uint64_t at, uint64_t len, int version, std::vector<Message>* out,
                   int depth) const {
  if (depth > kMaxDepth) fail("object header continuations nested too deeply");
  const uint8_t* p = ptr(at, len);
  spend(1 + len / 64);
  size_t o = 0;
  // version 2 headers carry their flags in the first byte of `version` (>> 8)
  const int v = version & 0xff, flags = version >> 8;
  while (true) {
    const size_t head = v == 1 ? 8 : 4 + ((flags & 4) ? 2 : 0);
    if (o + head > len) break;
    uint16_t type, size;
    if (v == 1) {
      type = (uint16_t)le(p + o, 2);
      size = (uint16_t)le(p + o + 2, 2);
    } else {
      type = p[o];
      size = (uint16_t)le(p + o + 1, 2);
    }
    o += head;
    if (o + size > len) fail("a header message overruns its block");
    if (type == 0x10) {  // continuation: more messages elsewhere
      need(0, (size_t)so_ + sl_, size, "continuation message");
      const uint64_t addr = le(p + o, so_), clen = le(p + o + so_, sl_);
      if (v == 1) {
        collect(addr, clen, version, out, depth + 1);
      } else {
        if (clen < 8 || memcmp(ptr(addr, 4), "OCHK", 4)) fail("bad continuation block");
        collect(addr + 4, clen - 8, version, out, depth + 1);
      }
    } else if (type != 0) {
      out->push_back({type, p + o, size});
    }
    o += size;
  }
}

std::vector<File::Message> File::messages(uint64_t h) const {
  std::vector<Message> out;
  const uint8_t* p = ptr(h, 16);
  if (!memcmp(p, "OHDR", 4)) {
    if (p[4] != 2) fail("object header version " + std::to_string(p[4]));
    const int flags = p[5];
    size_t o = 6;
    if (flags & 0x20) o += 16;  // the four times
    if (flags & 0x10) o += 4;   // attribute storage thresholds
    const int sz = 1 << (flags & 3);
    ptr(h, o + sz);
    const uint64_t len = uint_at(h + o, sz);
    o += sz;
    collect(h + o, len, 2 | (flags << 8), &out, 0);
  } else {
    if (p[0] != 1) fail("object header version " + std::to_string(p[0]));
    collect(h + 16, le(p + 8, 4), 1, &out, 0);
  }
  return out;
}

void File::group_btree(uint64_t btree, uint64_t heap, std::map<std::string, Link>* out,
                       std::vector<std::string>* order, int depth) const {
  if (depth > kMaxDepth) fail("group B-tree too deep");
  const uint8_t* hp = ptr(heap, 8 + 2 * (size_t)sl_ + so_);
  if (memcmp(hp, "HEAP", 4)) fail("bad local heap");
  const uint64_t hsize = le(hp + 8, sl_), hdata = le(hp + 8 + 2 * sl_, so_);
  const uint8_t* data = ptr(hdata, hsize);
  auto heap_str = [&](uint64_t off) {
    if (off >= hsize) fail("local heap offset out of range");
    spend(1 + (hsize - off) / 256);
    return std::string(reinterpret_cast<const char*>(data + off), strnlen(
        reinterpret_cast<const char*>(data + off), hsize - off));
  };
  const uint8_t* t = ptr(btree, 8 + 2 * (size_t)so_);
  if (memcmp(t, "TREE", 4) || t[4] != 0) fail("bad group B-tree node");
  const int level = t[5], used = (int)le(t + 6, 2);
  spend(1 + used);
  const size_t entry = (size_t)sl_ + so_;
  const uint8_t* k = ptr(btree + 8 + 2 * (size_t)so_, entry * used + sl_);
  for (int i = 0; i < used; ++i) {
    const uint64_t child = le(k + i * entry + sl_, so_);
    if (level > 0) {
      group_btree(child, heap, out, order, depth + 1);
      continue;
    }
    const uint8_t* sn = ptr(child, 8);
    if (memcmp(sn, "SNOD", 4)) fail("bad symbol-table node");
    const int nsym = (int)le(sn + 6, 2);
    spend(1 + nsym);
    const size_t es = 2 * (size_t)so_ + 24;
    const uint8_t* e = ptr(child + 8, es * nsym);
    for (int s = 0; s < nsym; ++s, e += es) {
      Link l;
      const std::string name = heap_str(le(e, so_));
      l.addr = le(e + so_, so_);
      if (le(e + 2 * so_, 4) == 2) {  // a soft link: its value in the heap
        l.soft = true;
        l.target = heap_str(le(e + 2 * so_ + 8, 4));
      }
      if (!out->count(name)) order->push_back(name);
      (*out)[name] = l;
    }
  }
}

std::map<std::string, File::Link> File::links(uint64_t header) const {
  std::map<std::string, Link> out;
  std::vector<std::string> order;
  for (const Message& m : messages(header)) {
    if (m.type == 0x11) {  // symbol table
      need(0, 2 * (size_t)so_, m.size, "symbol table message");
      group_btree(le(m.p, so_), le(m.p + so_, so_), &out, &order, 0);
    } else if (m.type == 0x06) {  // link
      const uint8_t* p = m.p;
      need(0, 2, m.size, "link message");
      const int flags = p[1];
      size_t o = 2;
      int ltype = 0;
      need(o, 1 + 8 + 1 + 8, m.size, "link message");
      if (flags & 8) ltype = p[o++];
      if (flags & 4) o += 8;
      if (flags & 16) o += 1;
      const int nb = 1 << (flags & 3);
      const size_t len = le(p + o, nb);
      o += nb;
      need(o, len, m.size, "link name");
      const std::string name(reinterpret_cast<const char*>(p + o), len);
      o += len;
      Link l;
      if (ltype == 0) {
        need(o, so_, m.size, "hard link");
        l.addr = le(p + o, so_);
      } else if (ltype == 1) {
        l.soft = true;
        need(o, 2, m.size, "soft link");
        const size_t tl = le(p + o, 2);
        need(o + 2, tl, m.size, "soft link value");
        l.target.assign(reinterpret_cast<const char*>(p + o + 2), tl);
      } else {
        continue;  // external links are not followed
      }
      if (!out.count(name)) order.push_back(name);
      out[name] = l;
    } else if (m.type == 0x02) {  // link info: a fractal heap means dense link storage
      need(0, 2 + 8 + (size_t)so_, m.size, "link info message");
      const int flags = m.p[1];
      const uint64_t heap = le(m.p + 2 + ((flags & 1) ? 8 : 0), so_);
      if (!undefined(heap, so_)) fail("groups in dense link storage are not read");
    }
  }
  return out;
}

std::vector<std::string> File::member_order(uint64_t header) const {
  std::map<std::string, Link> out;
  std::vector<std::string> order;
  for (const Message& m : messages(header)) {
    if (m.type == 0x11) {
      need(0, 2 * (size_t)so_, m.size, "symbol table message");
      group_btree(le(m.p, so_), le(m.p + so_, so_), &out, &order, 0);
    }
  }
  if (order.empty())
    for (auto& kv : links(header)) order.push_back(kv.first);
  return order;
}

uint64_t File::resolve(const std::string& path, int depth) const {
  if (depth > kMaxDepth) fail("soft links loop");
  uint64_t at = root_;
  size_t i = 0;
  while (i < path.size()) {
    while (i < path.size() && path[i] == '/') ++i;
    if (i >= path.size()) break;
    size_t j = path.find('/', i);
    if (j == std::string::npos) j = path.size();
    const std::string name = path.substr(i, j - i);
    const auto ls = links(at);
    const auto it = ls.find(name);
    if (it == ls.end()) fail("no member " + name + " in " + path.substr(0, i));
    if (it->second.soft) {
      const std::string& t = it->second.target;
      if (t.empty() || t[0] != '/') fail("relative soft link " + t);
      at = resolve(t, depth + 1);
    } else {
      at = it->second.addr;
    }
    i = j;
  }
  return at;
}

bool File::exists(const std::string& path) const {
  work_ = 0;
  try {
    resolve(path);
    return true;
  } catch (const std::runtime_error&) {
    return false;
  }
}

std::vector<std::string> File::members(const std::string& path) const {
  work_ = 0;
  return member_order(resolve(path));
}

Dataset File::dataset(const std::string& path) const {
  work_ = 0;
  const uint64_t h = resolve(path);
  Dataset d;
  bool have_space = false, have_type = false, have_layout = false;
  std::vector<Filter> filters;
  int layout = -1;
  uint64_t addr = 0, csize = 0;
  std::vector<uint64_t> chunk;
  const uint8_t* compact = nullptr;
  size_t compact_n = 0;
  for (const Message& m : messages(h)) {
    const uint8_t* p = m.p;
    if (m.type == 0x01) {  // dataspace
      need(0, 4, m.size, "dataspace");
      const int version = p[0], rank = p[1];
      size_t o = version == 1 ? 8 : 4;
      if (version == 2 && p[3] == 2) fail(path + " has a null dataspace");
      need(o, (size_t)rank * sl_, m.size, "dataspace");
      d.shape.clear();
      for (int k = 0; k < rank; ++k, o += sl_) d.shape.push_back(le(p + o, sl_));
      have_space = true;
    } else if (m.type == 0x03) {
      size_t u = 0;
      d.type = parse_type(p, m.size, &u);
      have_type = true;
    } else if (m.type == 0x0B) {
      filters = parse_filters(p, m.size);
    } else if (m.type == 0x08) {
      need(0, 3, m.size, "data layout");
      const int version = p[0];
      if (version == 3) {
        layout = p[1];
        if (layout == 0) {
          need(2, 2, m.size, "compact layout");
          compact_n = le(p + 2, 2);
          compact = p + 4;
          need(4, compact_n, m.size, "compact data");
        } else if (layout == 1) {
          need(2, (size_t)so_ + sl_, m.size, "contiguous layout");
          addr = le(p + 2, so_);
          csize = le(p + 2 + so_, sl_);
        } else if (layout == 2) {
          const int nd = p[2];
          need(3, (size_t)so_ + 4 * (size_t)nd, m.size, "chunked layout");
          addr = le(p + 3, so_);
          for (int k = 0; k < nd; ++k) chunk.push_back(le(p + 3 + so_ + 4 * k, 4));
        }
      } else if (version == 1 || version == 2) {
        const int nd = p[1];
        layout = p[2];
        size_t o = 8;
        need(o, (layout != 0 ? so_ : 0) + 4 * (size_t)nd + (layout == 0 ? 4 : 0), m.size,
             "data layout");
        if (layout != 0) {
          addr = le(p + o, so_);
          o += so_;
        }
        for (int k = 0; k < nd; ++k, o += 4) chunk.push_back(le(p + o, 4));
        if (layout == 0) {
          compact_n = le(p + o, 4);
          compact = p + o + 4;
          need(o + 4, compact_n, m.size, "compact data");
        } else if (layout == 1) {
          csize = 1;
          for (uint64_t c : chunk) csize *= c;
          chunk.clear();
        }
      } else {
        fail(path + ": data layout version " + std::to_string(version) + " is not read");
      }
      have_layout = true;
    }
  }
  if (!have_space || !have_type || !have_layout) fail(path + " is not a dataset");
  const size_t es = d.type.size;
  uint64_t total = es;
  for (uint64_t dim : d.shape) {
    if (dim != 0 && total > kMaxBytes / dim) fail(path + " is too large to read");
    total *= dim;
  }
  const uint64_t room = std::max<uint64_t>(buf_.size() * kMaxExpansion, 1u << 20);
  if (total > room) fail(path + " is larger than its file can hold");
  if (layout == 1 && !undefined(addr, so_)) ptr(addr, total);  // before any allocation
  d.bytes.assign(total, 0);
  if (layout == 0) {
    if (compact_n < total) fail(path + ": short compact data");
    if (total) std::memcpy(d.bytes.data(), compact, total);
  } else if (layout == 1) {
    if (!undefined(addr, so_) && total) {
      if (csize < total) fail(path + ": short contiguous data");
      std::memcpy(d.bytes.data(), ptr(addr, total), total);
    }
  } else if (layout == 2) {
    const size_t rank = d.shape.size();
    if (rank == 0 || chunk.size() != rank + 1) fail(path + ": chunk rank");
    uint64_t celems = 1;
    for (size_t k = 0; k < rank; ++k) {
      if (chunk[k] != 0 && celems > kMaxBytes / chunk[k]) fail(path + ": chunk too large");
      celems *= chunk[k];
    }
    if (celems != 0 && es > room / celems) fail(path + ": chunk larger than its file can hold");
    const uint64_t cbytes = celems * es;
    // Walk the chunk B-tree; decode and place every chunk.
    std::vector<std::pair<uint64_t, int>> stack;  // (node, depth)
    if (!undefined(addr, so_)) stack.push_back({addr, 0});
    const size_t key = 8 + 8 * (rank + 1);
    uint64_t visited = 0;
    while (!stack.empty()) {
      if (++visited > kMaxNodes) fail(path + ": chunk B-tree too large");
      const auto [node, depth] = stack.back();
      stack.pop_back();
      if (depth > kMaxDepth) fail(path + ": chunk B-tree too deep");
      const uint8_t* t = ptr(node, 8 + 2 * (size_t)so_);
      if (memcmp(t, "TREE", 4) || t[4] != 1) fail(path + ": bad chunk B-tree node");
      const int level = t[5], used = (int)le(t + 6, 2);
      spend(1 + used);
      const uint8_t* k = ptr(node + 8 + 2 * (size_t)so_, (key + so_) * used + key);
      for (int i = 0; i < used; ++i) {
        const uint8_t* kk = k + i * (key + so_);
        const uint64_t child = le(kk + key, so_);
        if (level > 0) {
          stack.push_back({child, depth + 1});
          continue;
        }
        const uint32_t stored = (uint32_t)le(kk, 4), mask = (uint32_t)le(kk + 4, 4);
        std::vector<uint64_t> off(rank);
        for (size_t r = 0; r < rank; ++r) off[r] = le(kk + 8 + 8 * r, 8);
        const uint8_t* src = ptr(child, stored);
        spend(1 + (cbytes + stored) / 65536);
        std::vector<uint8_t> c(src, src + stored);
        for (int fi = (int)filters.size() - 1; fi >= 0; --fi) {
          if (mask & (1u << fi)) continue;
          const Filter& f = filters[fi];
          if (f.id == 1) {
            c = inflate_all(c, cbytes);
          } else if (f.id == 2) {
            // the shuffle's element size is the datatype's (HDF5 stores it as client data)
            if (!f.values.empty() && f.values[0] != es)
              fail(path + ": shuffle element size differs from the datatype's");
            c = unshuffle(c, es);
          } else if (f.id == 3) {
            if (c.size() < 4) fail(path + ": short Fletcher-32 chunk");
            c.resize(c.size() - 4);
          } else {
            fail(path + ": filter " + std::to_string(f.id) + " is not read");
          }
        }
        if (c.size() < cbytes) fail(path + ": short chunk");
        // rows of the chunk's last dimension into place, clipped at the dataset's edges
        const uint64_t inner = chunk[rank - 1];
        std::vector<uint64_t> idx(rank, 0);
        for (uint64_t e = 0; e < celems; e += inner) {
          uint64_t dst = 0;
          bool inside = true;
          for (size_t r = 0; r < rank; ++r) {
            const uint64_t g = off[r] + idx[r];
            if (g >= d.shape[r]) inside = false;
            dst = dst * d.shape[r] + g;
          }
          if (inside) {
            const uint64_t n = std::min(inner, d.shape[rank - 1] - off[rank - 1]);
            std::memcpy(d.bytes.data() + dst * es, c.data() + e * es, n * es);
          }
          for (int r = (int)rank - 2; r >= 0; --r) {  // next row index
            if (++idx[r] < chunk[r]) break;
            idx[r] = 0;
          }
        }
      }
    }
  } else {
    fail(path + ": layout class " + std::to_string(layout));
  }
  return d;
}

}  // namespace ptyb::h5
