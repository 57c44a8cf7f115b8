// Minimal HDF5 reader / writer for the k-Wave file boundary.  The on-disk
// structures follow the published HDF5 File Format Specification (version
// 3.0): superblock, object headers and their messages, v1 B-trees, local
// heaps, symbol table nodes and the lookup3 metadata checksum.
#include "hdf5_lite.h"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <functional>

namespace h5 {

// ---------------------------------------------------------------------------
// lookup3 (Bob Jenkins, public domain): hashlittle() over a byte string
// ---------------------------------------------------------------------------
static inline uint32_t rotl(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }

uint32_t lookup3(const void* key, size_t length, uint32_t initval) {
  const uint8_t* k = static_cast<const uint8_t*>(key);
  uint32_t a, b, c;
  a = b = c = 0xdeadbeefu + static_cast<uint32_t>(length) + initval;
  auto w = [&](int i) { return static_cast<uint32_t>(k[i]); };
  while (length > 12) {
    a += w(0) | (w(1) << 8) | (w(2) << 16) | (w(3) << 24);
    b += w(4) | (w(5) << 8) | (w(6) << 16) | (w(7) << 24);
    c += w(8) | (w(9) << 8) | (w(10) << 16) | (w(11) << 24);
    a -= c; a ^= rotl(c, 4); c += b;
    b -= a; b ^= rotl(a, 6); a += c;
    c -= b; c ^= rotl(b, 8); b += a;
    a -= c; a ^= rotl(c, 16); c += b;
    b -= a; b ^= rotl(a, 19); a += c;
    c -= b; c ^= rotl(b, 4); b += a;
    length -= 12;
    k += 12;
  }
  switch (length) {
    case 12: c += w(11) << 24; [[fallthrough]];
    case 11: c += w(10) << 16; [[fallthrough]];
    case 10: c += w(9) << 8; [[fallthrough]];
    case 9: c += w(8); [[fallthrough]];
    case 8: b += w(7) << 24; [[fallthrough]];
    case 7: b += w(6) << 16; [[fallthrough]];
    case 6: b += w(5) << 8; [[fallthrough]];
    case 5: b += w(4); [[fallthrough]];
    case 4: a += w(3) << 24; [[fallthrough]];
    case 3: a += w(2) << 16; [[fallthrough]];
    case 2: a += w(1) << 8; [[fallthrough]];
    case 1: a += w(0); break;
    case 0: return c;
  }
  c ^= b; c -= rotl(b, 14);
  a ^= c; a -= rotl(c, 11);
  b ^= a; b -= rotl(a, 25);
  c ^= b; c -= rotl(b, 16);
  a ^= c; a -= rotl(c, 4);
  b ^= a; b -= rotl(a, 14);
  c ^= b; c -= rotl(b, 24);
  return c;
}

// ---------------------------------------------------------------------------
// reader
// ---------------------------------------------------------------------------
namespace {
struct Msg {
  unsigned type;
  const uint8_t* data;
  size_t size;
};

struct Filter {
  unsigned id;
  std::vector<uint32_t> cd;
};

struct Layout {
  int cls = -1;  // 0 compact, 1 contiguous, 2 chunked
  uint64_t addr = 0, size = 0;
  const uint8_t* compact = nullptr;
  std::vector<uint64_t> chunk;  // chunk dims (without the element dimension)
  int version = 3;
  int index_type = 0;  // layout v4 chunk index (1: single chunk)
  uint64_t single_size = 0;
  uint32_t single_mask = 0;
};
}  // namespace

struct Reader::Impl {
  int fd = -1;
  const uint8_t* map = nullptr;
  size_t fsize = 0;
  uint64_t base = 0;  // absolute offset of address 0
  int so = 8, sl = 8;
  uint64_t root = 0;

  ~Impl() {
    if (map) munmap(const_cast<uint8_t*>(map), fsize);
    if (fd >= 0) close(fd);
  }
  const uint8_t* at(uint64_t addr, uint64_t n) const {
    const uint64_t off = base + addr;
    if (off < base || off + n > fsize || off + n < off) throw Error("address out of range (truncated file?)");
    return map + off;
  }
  static uint64_t le(const uint8_t* p, int n) {
    uint64_t v = 0;
    for (int i = n - 1; i >= 0; --i) v = (v << 8) | p[i];
    return v;
  }
  bool undef(uint64_t a) const { return so == 8 ? a == ~0ull : a == ((1ull << (8 * so)) - 1); }

  void open_file(const std::string& path) {
    fd = ::open(path.c_str(), O_RDONLY);
    if (fd < 0) throw Error("cannot open " + path);
    struct stat st;
    if (fstat(fd, &st) != 0) throw Error("cannot stat " + path);
    fsize = (size_t)st.st_size;
    if (fsize < 64) throw Error("file too small to be HDF5: " + path);
    void* m = mmap(nullptr, fsize, PROT_READ, MAP_PRIVATE, fd, 0);
    if (m == MAP_FAILED) throw Error("cannot map " + path);
    map = static_cast<const uint8_t*>(m);
    static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    uint64_t sb = ~0ull;
    for (uint64_t o = 0; o + 8 <= fsize; o = (o == 0 ? 512 : o * 2))
      if (std::memcmp(map + o, sig, 8) == 0) {
        sb = o;
        break;
      }
    if (sb == ~0ull) throw Error("no HDF5 superblock in " + path);
    const uint8_t* p = map + sb;
    const int ver = p[8];
    base = sb;  // addresses are relative to the superblock (user-block files)
    if (ver == 0 || ver == 1) {
      so = p[13];
      sl = p[14];
      const int extra = (ver == 1) ? 4 : 0;
      const uint8_t* q = p + 24 + extra;
      const uint64_t base_addr = le(q, so);
      if (base_addr != 0 && base_addr != sb) base = base_addr;
      q += 4 * so;               // base, free space, end of file, driver info
      root = le(q + so, so);     // root symbol table entry: name offset, header address
    } else if (ver == 2 || ver == 3) {
      so = p[9];
      sl = p[10];
      const uint8_t* q = p + 12;
      const uint64_t base_addr = le(q, so);
      if (base_addr != 0 && base_addr != sb) base = base_addr;
      root = le(q + 3 * so, so);
    } else {
      throw Error("unsupported superblock version " + std::to_string(ver));
    }
  }

  std::vector<Msg> messages(uint64_t addr) {
    std::vector<Msg> out;
    const uint8_t* p = at(addr, 16);
    struct Block {
      uint64_t addr, len;
      bool first;
    };
    std::vector<Block> blocks;
    if (std::memcmp(p, "OHDR", 4) == 0) {
      const int flags = p[5];
      size_t off = 6;
      if (flags & 0x20) off += 16;
      if (flags & 0x10) off += 4;
      const int nb = 1 << (flags & 3);
      const uint64_t len = le(at(addr + off, nb), nb);
      off += nb;
      const bool crt = flags & 0x04;
      blocks.push_back({addr + off, len, true});
      for (size_t bi = 0; bi < blocks.size(); ++bi) {
        Block b = blocks[bi];
        uint64_t a = b.addr, end = b.addr + b.len;
        if (!b.first) {
          if (std::memcmp(at(a, 4), "OCHK", 4) != 0) throw Error("bad continuation block");
          a += 4;
          end = b.addr + b.len - 4;
        }
        while (a + 4 <= end) {
          const uint8_t* m = at(a, 4);
          const unsigned type = m[0];
          const size_t size = le(m + 1, 2);
          const size_t hdr = 4 + (crt ? 2 : 0);
          if (a + hdr + size > end) break;
          const uint8_t* d = at(a + hdr, size);
          if (type == 0x10) {
            blocks.push_back({le(d, so), le(d + so, sl), false});
          } else if (type != 0) {
            out.push_back({type, d, size});
          }
          a += hdr + size;
        }
      }
    } else if (p[0] == 1) {
      const unsigned nmsg = (unsigned)le(p + 2, 2);
      const uint64_t len = le(p + 8, 4);
      blocks.push_back({addr + 16, len, true});
      unsigned count = 0;
      for (size_t bi = 0; bi < blocks.size() && count < nmsg; ++bi) {
        uint64_t a = blocks[bi].addr;
        const uint64_t end = blocks[bi].addr + blocks[bi].len;
        while (a + 8 <= end && count < nmsg) {
          const uint8_t* m = at(a, 8);
          const unsigned type = (unsigned)le(m, 2);
          const size_t size = le(m + 2, 2);
          const uint8_t* d = at(a + 8, size);
          ++count;
          if (type == 0x10)
            blocks.push_back({le(d, so), le(d + so, sl), false});
          else if (type != 0)
            out.push_back({type, d, size});
          a += 8 + size;
        }
      }
    } else {
      throw Error("unsupported object header");
    }
    return out;
  }

  // children of a symbol-table group: walk the v1 B-tree of SNOD leaves
  void symtab_children(uint64_t btree, uint64_t heap, std::map<std::string, uint64_t>& out) {
    const uint8_t* h = at(heap, 32);
    if (std::memcmp(h, "HEAP", 4) != 0) throw Error("bad local heap");
    const uint64_t seg_size = le(h + 8, sl);
    const uint64_t seg = le(h + 8 + 2 * sl, so);
    const uint8_t* names = at(seg, seg_size);
    std::function<void(uint64_t)> walk = [&](uint64_t node) {
      const uint8_t* b = at(node, 8 + 2 * so);
      if (std::memcmp(b, "TREE", 4) != 0) throw Error("bad group B-tree node");
      const int level = b[5];
      const unsigned n = (unsigned)le(b + 6, 2);
      const uint8_t* q = at(node + 8 + 2 * so, (uint64_t)(n + 1) * sl + (uint64_t)n * so);
      for (unsigned i = 0; i < n; ++i) {
        const uint64_t child = le(q + sl + (uint64_t)i * (sl + so), so);
        if (level > 0) {
          walk(child);
        } else {
          const uint8_t* s = at(child, 8);
          if (std::memcmp(s, "SNOD", 4) != 0) throw Error("bad symbol table node");
          const unsigned ns = (unsigned)le(s + 6, 2);
          const uint64_t esz = 2 * so + 24;
          const uint8_t* e = at(child + 8, ns * esz);
          for (unsigned j = 0; j < ns; ++j) {
            const uint64_t noff = le(e + j * esz, so);
            const uint64_t oh = le(e + j * esz + so, so);
            if (noff >= seg_size) throw Error("bad link name offset");
            out[std::string(reinterpret_cast<const char*>(names + noff))] = oh;
          }
        }
      }
    };
    walk(btree);
  }

  std::map<std::string, uint64_t> children(uint64_t oh) {
    std::map<std::string, uint64_t> out;
    for (const Msg& m : messages(oh)) {
      if (m.type == 0x11) {
        symtab_children(le(m.data, so), le(m.data + so, so), out);
      } else if (m.type == 0x06) {
        const uint8_t* d = m.data;
        const int flags = d[1];
        size_t off = 2;
        int ltype = 0;
        if (flags & 0x08) ltype = d[off++];
        if (flags & 0x04) off += 8;
        if (flags & 0x10) off += 1;
        const int nb = 1 << (flags & 3);
        const size_t nlen = le(d + off, nb);
        off += nb;
        std::string name(reinterpret_cast<const char*>(d + off), nlen);
        off += nlen;
        if (ltype == 0) out[name] = le(d + off, so);
      } else if (m.type == 0x02) {
        const int flags = m.data[1];
        const uint64_t fh = le(m.data + 2 + ((flags & 1) ? 8 : 0), so);
        if (!undef(fh)) throw Error("groups with dense link storage are not supported");
      }
    }
    return out;
  }

  uint64_t lookup(const std::string& path) {
    uint64_t oh = root;
    size_t i = 0;
    while (i < path.size()) {
      while (i < path.size() && path[i] == '/') ++i;
      if (i >= path.size()) break;
      size_t j = path.find('/', i);
      if (j == std::string::npos) j = path.size();
      const std::string name = path.substr(i, j - i);
      auto ch = children(oh);
      auto it = ch.find(name);
      if (it == ch.end()) throw Error("no object " + path);
      oh = it->second;
      i = j;
    }
    return oh;
  }

  TypeInfo parse_type(const uint8_t* d) {
    TypeInfo t;
    const int cls = d[0] & 0x0f;
    t.size = (int)le(d + 4, 4);
    if (cls == 0) {
      t.kind = Kind::Int;
      t.big_endian = d[1] & 1;
      t.sign = d[1] & 0x08;
    } else if (cls == 1) {
      t.kind = Kind::Float;
      t.big_endian = d[1] & 1;
    } else if (cls == 3) {
      t.kind = Kind::String;
    }
    return t;
  }

  std::vector<uint64_t> parse_space(const uint8_t* d) {
    const int ver = d[0], rank = d[1];
    const uint8_t* q = (ver == 1) ? d + 8 : d + 4;
    std::vector<uint64_t> dims(rank);
    for (int i = 0; i < rank; ++i) dims[i] = le(q + (size_t)i * sl, sl);
    return dims;
  }

  void dataset(uint64_t oh, DatasetInfo& info, Layout& lay, std::vector<Filter>& filters) {
    bool have_space = false, have_type = false;
    for (const Msg& m : messages(oh)) {
      const uint8_t* d = m.data;
      if (m.type == 0x01) {
        info.dims = parse_space(d);
        have_space = true;
      } else if (m.type == 0x03) {
        info.type = parse_type(d);
        have_type = true;
      } else if (m.type == 0x08) {
        lay.version = d[0];
        if (d[0] == 3 || d[0] == 4) {
          lay.cls = d[1];
          if (lay.cls == 0) {
            lay.size = le(d + 2, 2);
            lay.compact = d + 4;
          } else if (lay.cls == 1) {
            lay.addr = le(d + 2, so);
            lay.size = le(d + 2 + so, sl);
          } else if (lay.cls == 2 && d[0] == 3) {
            const int nd = d[2];
            lay.addr = le(d + 3, so);
            for (int i = 0; i < nd - 1; ++i) lay.chunk.push_back(le(d + 3 + so + 4 * i, 4));
          } else if (lay.cls == 2 && d[0] == 4) {
            const int flags = d[2], nd = d[3], enc = d[4];
            size_t off = 5;
            for (int i = 0; i < nd; ++i, off += enc)
              if (i < nd - 1) lay.chunk.push_back(le(d + off, enc));
            lay.index_type = d[off++];
            if (lay.index_type != 1) throw Error("unsupported chunk index type " + std::to_string(lay.index_type));
            if (flags & 0x02) {
              lay.single_size = le(d + off, sl);
              lay.single_mask = (uint32_t)le(d + off + sl, 4);
              off += sl + 4;
            }
            lay.addr = le(d + off, so);
          } else {
            throw Error("unsupported data layout");
          }
        } else if (d[0] == 1 || d[0] == 2) {
          const int nd = d[1];
          lay.cls = d[2];
          size_t off = 8;
          if (lay.cls != 0) {
            lay.addr = le(d + off, so);
            off += so;
          }
          std::vector<uint64_t> dd;
          for (int i = 0; i < nd; ++i) dd.push_back(le(d + off + 4 * i, 4));
          off += 4 * nd;
          if (lay.cls == 2) {
            dd.pop_back();
            lay.chunk = dd;
          } else if (lay.cls == 0) {
            lay.size = le(d + off, 4);
            lay.compact = d + off + 4;
          } else {
            uint64_t n = 1;
            for (auto v : dd) n *= v;
            lay.size = n;
          }
        } else {
          throw Error("unsupported data layout version");
        }
      } else if (m.type == 0x0B) {
        const int ver = d[0], n = d[1];
        size_t off = (ver == 1) ? 8 : 2;
        for (int i = 0; i < n; ++i) {
          Filter f;
          f.id = (unsigned)le(d + off, 2);
          off += 2;
          size_t nlen = 0;
          if (ver == 1 || f.id >= 256) {
            nlen = le(d + off, 2);
            off += 2;
          }
          off += 2;  // flags
          const unsigned ncd = (unsigned)le(d + off, 2);
          off += 2;
          if (ver == 1) nlen = (nlen + 7) / 8 * 8;
          off += nlen;
          for (unsigned c = 0; c < ncd; ++c, off += 4) f.cd.push_back((uint32_t)le(d + off, 4));
          if (ver == 1 && (ncd & 1)) off += 4;
          filters.push_back(f);
        }
      }
    }
    if (!have_space || !have_type || lay.cls < 0) throw Error("object is not a dataset");
  }

  std::vector<uint8_t> unfilter(const uint8_t* src, size_t n, uint32_t mask, const std::vector<Filter>& filters,
                                size_t expect, int elem) {
    std::vector<uint8_t> buf(src, src + n);
    for (int i = (int)filters.size() - 1; i >= 0; --i) {
      if (mask & (1u << i)) continue;
      const Filter& f = filters[i];
      if (f.id == 1) {  // deflate
        std::vector<uint8_t> out(expect);
        uLongf dl = (uLongf)expect;
        if (uncompress(out.data(), &dl, buf.data(), (uLong)buf.size()) != Z_OK)
          throw Error("deflate stream corrupt");
        out.resize(dl);
        buf.swap(out);
      } else if (f.id == 2) {  // shuffle
        const int es = f.cd.empty() ? elem : (int)f.cd[0];
        std::vector<uint8_t> out(buf.size());
        const size_t ne = buf.size() / es;
        for (int b = 0; b < es; ++b)
          for (size_t e = 0; e < ne; ++e) out[e * es + b] = buf[b * ne + e];
        buf.swap(out);
      } else if (f.id == 3) {  // fletcher32: drop the trailing checksum
        if (buf.size() >= 4) buf.resize(buf.size() - 4);
      } else {
        throw Error("unsupported filter " + std::to_string(f.id));
      }
    }
    return buf;
  }

  // raw element bytes of a dataset in C order
  std::vector<uint8_t> raw(const std::string& path, DatasetInfo& info) {
    Layout lay;
    std::vector<Filter> filters;
    dataset(lookup(path), info, lay, filters);
    const size_t es = (size_t)info.type.size;
    const uint64_t n = info.numel();
    std::vector<uint8_t> out(n * es, 0);
    if (n == 0) return out;
    if (lay.cls == 0) {
      std::memcpy(out.data(), lay.compact, std::min<uint64_t>(lay.size, out.size()));
    } else if (lay.cls == 1) {
      if (undef(lay.addr)) return out;  // never written: fill value 0
      std::memcpy(out.data(), at(lay.addr, n * es), n * es);
    } else {
      const int rank = (int)info.dims.size();
      if ((int)lay.chunk.size() != rank) throw Error("chunk rank mismatch");
      uint64_t cn = 1;
      for (auto c : lay.chunk) cn *= c;
      auto place = [&](const uint8_t* src, const std::vector<uint64_t>& off) {
        std::vector<uint64_t> idx(rank, 0);
        for (uint64_t e = 0; e < cn; ++e) {
          uint64_t lin = 0;
          bool inside = true;
          for (int r = 0; r < rank; ++r) {
            const uint64_t g = off[r] + idx[r];
            if (g >= info.dims[r]) {
              inside = false;
              break;
            }
            lin = lin * info.dims[r] + g;
          }
          if (inside) std::memcpy(&out[lin * es], src + e * es, es);
          for (int r = rank - 1; r >= 0; --r) {
            if (++idx[r] < lay.chunk[r]) break;
            idx[r] = 0;
          }
        }
      };
      if (lay.version == 4) {
        std::vector<uint64_t> off(rank, 0);
        const uint64_t sz = lay.single_size ? lay.single_size : cn * es;
        auto b = unfilter(at(lay.addr, sz), sz, lay.single_mask, filters, cn * es, (int)es);
        if (b.size() < cn * es) throw Error("short chunk");
        place(b.data(), off);
      } else {
        std::function<void(uint64_t)> walk = [&](uint64_t node) {
          const uint8_t* b = at(node, 8 + 2 * so);
          if (std::memcmp(b, "TREE", 4) != 0 || b[4] != 1) throw Error("bad chunk B-tree node");
          const int level = b[5];
          const unsigned ne = (unsigned)le(b + 6, 2);
          const uint64_t ksz = 8 + 8ull * (rank + 1);
          const uint8_t* q = at(node + 8 + 2 * so, (ne + 1) * ksz + ne * so);
          for (unsigned i = 0; i < ne; ++i) {
            const uint8_t* key = q + i * (ksz + so);
            const uint64_t child = le(key + ksz, so);
            if (level > 0) {
              walk(child);
              continue;
            }
            const uint32_t csize = (uint32_t)le(key, 4);
            const uint32_t mask = (uint32_t)le(key + 4, 4);
            std::vector<uint64_t> off(rank);
            for (int r = 0; r < rank; ++r) off[r] = le(key + 8 + 8 * r, 8);
            auto data = unfilter(at(child, csize), csize, mask, filters, cn * es, (int)es);
            if (data.size() < cn * es) throw Error("short chunk");
            place(data.data(), off);
          }
        };
        if (!undef(lay.addr)) walk(lay.addr);
      }
    }
    if (info.type.big_endian && es > 1)
      for (uint64_t e = 0; e < n; ++e) std::reverse(&out[e * es], &out[e * es] + es);
    return out;
  }

  template <class T>
  std::vector<T> convert(const std::string& path) {
    DatasetInfo info;
    auto b = raw(path, info);
    const uint64_t n = info.numel();
    std::vector<T> v(n);
    const TypeInfo& t = info.type;
    for (uint64_t i = 0; i < n; ++i) {
      const uint8_t* p = &b[i * t.size];
      if (t.kind == Kind::Float && t.size == 4) {
        float f;
        std::memcpy(&f, p, 4);
        v[i] = (T)f;
      } else if (t.kind == Kind::Float && t.size == 8) {
        double f;
        std::memcpy(&f, p, 8);
        v[i] = (T)f;
      } else if (t.kind == Kind::Int) {
        uint64_t u = le(p, t.size);
        if (t.sign && t.size < 8 && (u >> (8 * t.size - 1)) & 1) u |= ~0ull << (8 * t.size);
        v[i] = t.sign ? (T)(int64_t)u : (T)u;
      } else {
        throw Error(path + " is not numeric");
      }
    }
    return v;
  }
};

Reader::Reader(const std::string& path) : p_(new Impl) { p_->open_file(path); }
Reader::~Reader() = default;

bool Reader::exists(const std::string& path) {
  try {
    p_->lookup(path);
    return true;
  } catch (const Error&) {
    return false;
  }
}

DatasetInfo Reader::info(const std::string& path) {
  DatasetInfo info;
  Layout lay;
  std::vector<Filter> f;
  p_->dataset(p_->lookup(path), info, lay, f);
  return info;
}

std::vector<float> Reader::read_float(const std::string& path) { return p_->convert<float>(path); }
std::vector<double> Reader::read_double(const std::string& path) { return p_->convert<double>(path); }
std::vector<uint64_t> Reader::read_u64(const std::string& path) { return p_->convert<uint64_t>(path); }

std::string Reader::attribute_string(const std::string& path, const std::string& name) {
  for (const Msg& m : p_->messages(p_->lookup(path))) {
    if (m.type != 0x0C) continue;
    const uint8_t* d = m.data;
    const int ver = d[0];
    const size_t nsz = Impl::le(d + 2, 2), tsz = Impl::le(d + 4, 2), ssz = Impl::le(d + 6, 2);
    size_t off = (ver == 3) ? 9 : 8;
    auto pad = [&](size_t v) { return ver == 1 ? (v + 7) / 8 * 8 : v; };
    std::string an(reinterpret_cast<const char*>(d + off));
    off += pad(nsz);
    const uint8_t* t = d + off;
    off += pad(tsz) + pad(ssz);
    if (an != name) continue;
    if ((t[0] & 0x0f) != 3) return "";
    const size_t len = Impl::le(t + 4, 4);
    std::string s(reinterpret_cast<const char*>(d + off), std::min(len, m.size - off));
    const size_t z = s.find('\0');
    if (z != std::string::npos) s.resize(z);
    while (!s.empty() && s.back() == ' ') s.pop_back();
    return s;
  }
  return "";
}

// ---------------------------------------------------------------------------
// writer
// ---------------------------------------------------------------------------
namespace {
struct Buf {
  std::vector<uint8_t> b;
  void u8(unsigned v) { b.push_back((uint8_t)v); }
  void u16(unsigned v) { put(v, 2); }
  void u32(uint64_t v) { put(v, 4); }
  void u64(uint64_t v) { put(v, 8); }
  void put(uint64_t v, int n) {
    for (int i = 0; i < n; ++i) b.push_back((uint8_t)(v >> (8 * i)));
  }
  void bytes(const void* p, size_t n) {
    const uint8_t* q = static_cast<const uint8_t*>(p);
    b.insert(b.end(), q, q + n);
  }
  void str(const std::string& s) { bytes(s.data(), s.size()); }
};

const uint64_t kUndef = ~0ull;

void message(Buf& out, unsigned type, const Buf& body) {
  out.u8(type);
  out.u16((unsigned)body.b.size());
  out.u8(0);
  out.bytes(body.b.data(), body.b.size());
}

Buf string_type(size_t len) {
  Buf t;
  t.u8(0x13);  // version 1, class 3 (string)
  t.u8(0x00);  // null-terminated, ASCII
  t.u8(0);
  t.u8(0);
  t.u32(len);
  return t;
}

Buf attribute_msg(const std::string& name, const std::string& value) {
  Buf a;
  const Buf t = string_type(value.size() + 1);
  Buf sp;
  sp.u8(2);  // dataspace version 2, scalar
  sp.u8(0);
  sp.u8(0);
  sp.u8(0);
  a.u8(3);  // attribute message version 3
  a.u8(0);
  a.u16((unsigned)name.size() + 1);
  a.u16((unsigned)t.b.size());
  a.u16((unsigned)sp.b.size());
  a.u8(0);  // ASCII name
  a.str(name);
  a.u8(0);
  a.bytes(t.b.data(), t.b.size());
  a.bytes(sp.b.data(), sp.b.size());
  a.str(value);
  a.u8(0);
  return a;
}

Buf ohdr(const Buf& msgs) {
  Buf h;
  h.str("OHDR");
  h.u8(2);     // version
  h.u8(0x02);  // chunk-0 size stored in 4 bytes
  h.u32(msgs.b.size());
  h.bytes(msgs.b.data(), msgs.b.size());
  h.u32(lookup3(h.b.data(), h.b.size(), 0));
  return h;
}

size_t dtype_size(DType t) { return t == DType::F32 ? 4 : 8; }

Buf dtype_msg(DType t) {
  Buf d;
  if (t == DType::U64) {
    d.u8(0x10);  // version 1, class 0 (fixed point)
    d.u8(0x00);  // little endian, unsigned
    d.u8(0);
    d.u8(0);
    d.u32(8);
    d.u16(0);   // bit offset
    d.u16(64);  // precision
  } else {
    const bool f32 = t == DType::F32;
    d.u8(0x11);        // version 1, class 1 (floating point)
    d.u8(0x20);        // little endian, implied mantissa MSB
    d.u8(f32 ? 31 : 63);  // sign bit position
    d.u8(0);
    d.u32(f32 ? 4 : 8);
    d.u16(0);               // bit offset
    d.u16(f32 ? 32 : 64);   // precision
    d.u8(f32 ? 23 : 52);    // exponent location
    d.u8(f32 ? 8 : 11);     // exponent size
    d.u8(0);                // mantissa location
    d.u8(f32 ? 23 : 52);    // mantissa size
    d.u32(f32 ? 127 : 1023);  // exponent bias
  }
  return d;
}
}  // namespace

Writer::Node* Writer::group(const std::string& path, std::string* leaf) {
  Node* g = &root_;
  size_t i = 0;
  std::vector<std::string> parts;
  while (i < path.size()) {
    while (i < path.size() && path[i] == '/') ++i;
    size_t j = path.find('/', i);
    if (j == std::string::npos) j = path.size();
    if (j > i) parts.push_back(path.substr(i, j - i));
    i = j;
  }
  if (parts.empty()) throw Error("empty dataset path");
  for (size_t k = 0; k + 1 < parts.size(); ++k) {
    auto it = g->children.find(parts[k]);
    if (it == g->children.end()) {
      g->order.push_back(parts[k]);
      it = g->children.emplace(parts[k], std::make_unique<Node>()).first;
    }
    if (!it->second->is_group) throw Error(parts[k] + " is a dataset");
    g = it->second.get();
  }
  *leaf = parts.back();
  return g;
}

void Writer::dataset(const std::string& path, DType t, const std::vector<uint64_t>& dims, const void* data,
                     const std::map<std::string, std::string>& attrs) {
  std::string leaf;
  Node* g = group(path, &leaf);
  if (g->children.count(leaf)) throw Error("duplicate object " + path);
  auto n = std::make_unique<Node>();
  n->is_group = false;
  n->type = t;
  n->dims = dims;
  n->data = data;
  n->attrs = attrs;
  g->order.push_back(leaf);
  g->children.emplace(leaf, std::move(n));
}

void Writer::root_attribute(const std::string& name, const std::string& value) { root_.attrs[name] = value; }

void Writer::write(const std::string& file) {
  // serialise headers: datasets get fixed-size headers, groups depend on
  // their children's addresses, so lay out in two passes
  const uint64_t sb_size = 48;
  std::vector<Node*> all;
  std::function<void(Node*)> collect = [&](Node* n) {
    all.push_back(n);
    for (auto& name : n->order) collect(n->children[name].get());
  };
  collect(&root_);
  auto dataset_header = [&](Node* n) {
    Buf m, body;
    body.u8(2);
    body.u8((unsigned)n->dims.size());
    body.u8(0);
    body.u8(1);  // simple dataspace
    for (auto v : n->dims) body.u64(v);
    message(m, 0x01, body);
    message(m, 0x03, dtype_msg(n->type));
    Buf fill;
    fill.u8(2);  // fill value message version 2
    fill.u8(1);  // allocate early
    fill.u8(1);  // never write fill values
    fill.u8(0);  // no fill value defined
    message(m, 0x05, fill);
    uint64_t bytes = dtype_size(n->type);
    for (auto v : n->dims) bytes *= v;
    Buf lay;
    lay.u8(3);
    lay.u8(1);  // contiguous
    lay.u64(n->data_addr);
    lay.u64(bytes);
    message(m, 0x08, lay);
    for (auto& kv : n->attrs) message(m, 0x0C, attribute_msg(kv.first, kv.second));
    return ohdr(m);
  };
  auto group_header = [&](Node* n) {
    Buf m, li, gi;
    li.u8(0);
    li.u8(0);
    li.u64(kUndef);  // no fractal heap: links are stored compactly
    li.u64(kUndef);
    message(m, 0x02, li);
    gi.u8(0);
    gi.u8(0);
    message(m, 0x0A, gi);
    for (auto& name : n->order) {
      Buf l;
      l.u8(1);     // link message version 1
      l.u8(0x00);  // 1-byte name length, hard link
      l.u8((unsigned)name.size());
      l.str(name);
      l.u64(n->children[name]->addr);
      message(m, 0x06, l);
    }
    for (auto& kv : n->attrs) message(m, 0x0C, attribute_msg(kv.first, kv.second));
    return ohdr(m);
  };
  // pass 1: sizes (addresses do not change the header sizes)
  uint64_t cur = sb_size;
  for (Node* n : all) {
    n->header_size = n->is_group ? group_header(n).b.size() : dataset_header(n).b.size();
    n->addr = cur;
    cur += n->header_size;
  }
  for (Node* n : all) {
    if (n->is_group) continue;
    uint64_t bytes = dtype_size(n->type);
    for (auto v : n->dims) bytes *= v;
    cur = (cur + 7) / 8 * 8;
    n->data_addr = cur;
    cur += bytes;
  }
  const uint64_t eof = cur;
  FILE* f = std::fopen(file.c_str(), "wb");
  if (!f) throw Error("cannot create " + file);
  auto fail = [&](const char* what) {
    std::fclose(f);
    std::remove(file.c_str());
    throw Error(std::string(what) + " " + file);
  };
  Buf sb;
  const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  sb.bytes(sig, 8);
  sb.u8(2);
  sb.u8(8);
  sb.u8(8);
  sb.u8(0);
  sb.u64(0);       // base address
  sb.u64(kUndef);  // no superblock extension
  sb.u64(eof);
  sb.u64(root_.addr);
  sb.u32(lookup3(sb.b.data(), sb.b.size(), 0));
  if (std::fwrite(sb.b.data(), 1, sb.b.size(), f) != sb.b.size()) fail("write failed:");
  for (Node* n : all) {
    const Buf h = n->is_group ? group_header(n) : dataset_header(n);
    if (h.b.size() != n->header_size) fail("header size changed:");
    if (std::fwrite(h.b.data(), 1, h.b.size(), f) != h.b.size()) fail("write failed:");
  }
  uint64_t pos = sb_size;
  for (Node* n : all) pos += n->header_size;
  for (Node* n : all) {
    if (n->is_group) continue;
    static const uint8_t zeros[8] = {0};
    if (n->data_addr > pos) {
      if (std::fwrite(zeros, 1, n->data_addr - pos, f) != n->data_addr - pos) fail("write failed:");
      pos = n->data_addr;
    }
    uint64_t bytes = dtype_size(n->type);
    for (auto v : n->dims) bytes *= v;
    if (bytes && std::fwrite(n->data, 1, bytes, f) != bytes) fail("write failed:");
    pos += bytes;
  }
  if (std::fclose(f) != 0) {
    std::remove(file.c_str());
    throw Error("close failed: " + file);
  }
}

}  // namespace h5

// test hook: the metadata checksum, exported for known-answer tests
extern "C" uint32_t kwb_h5_lookup3(const void* key, size_t length, uint32_t initval) {
  return h5::lookup3(key, length, initval);
}

// Test hooks (not part of the public header): read one dataset converted to
// double, and write one float / uint64 dataset, so the reader and writer can
// be checked against independent implementations without a GPU.
// kwb_h5_read returns the element count (0 .. cap), or -1 with `err` filled.
extern "C" int64_t kwb_h5_read(const char* file, const char* path, double* out, uint64_t cap, uint64_t* dims,
                               int* rank, char* err, int errlen) {
  try {
    h5::Reader r(file);
    h5::DatasetInfo di = r.info(path);
    *rank = (int)di.dims.size();
    for (size_t i = 0; i < di.dims.size() && i < 8; ++i) dims[i] = di.dims[i];
    std::vector<double> v = r.read_double(path);
    if (v.size() > cap) throw h5::Error("buffer too small");
    std::copy(v.begin(), v.end(), out);
    return (int64_t)v.size();
  } catch (const std::exception& e) {
    snprintf(err, errlen, "%s", e.what());
    return -1;
  }
}

extern "C" int64_t kwb_h5_read_attribute(const char* file, const char* path, const char* name, char* out,
                                         int outlen) {
  try {
    h5::Reader r(file);
    snprintf(out, outlen, "%s", r.attribute_string(path, name).c_str());
    return 0;
  } catch (const std::exception& e) {
    snprintf(out, outlen, "%s", e.what());
    return -1;
  }
}

extern "C" int kwb_h5_write(const char* file, int n, const char* const* paths, const int* types,
                            const uint64_t* const* dims, const int* ranks, const void* const* data, char* err,
                            int errlen) {
  try {
    h5::Writer w;
    for (int i = 0; i < n; ++i) {
      std::vector<uint64_t> d(dims[i], dims[i] + ranks[i]);
      h5::DType t = types[i] == 0 ? h5::DType::F32 : types[i] == 1 ? h5::DType::F64 : h5::DType::U64;
      w.dataset(paths[i], t, d, data[i], {{"data_type", types[i] == 2 ? "long" : "float"}, {"domain_type", "real"}});
    }
    w.root_attribute("file_type", "output");
    w.write(file);
    return 0;
  } catch (const std::exception& e) {
    snprintf(err, errlen, "%s", e.what());
    return -1;
  }
}
