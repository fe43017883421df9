// Restart files in the reference's HDF5 layout, written and read without the HDF5 library.
//
// The container code implements the subset of the published HDF5 File Format Specification
// (version 3.0, The HDF Group) that the reference's continua files use when its HDF5 library
// runs with default property lists (h5tools/HdfRoutines.F90:11-96, :428-600): a version-0
// superblock, a root group stored as a symbol table (version-1 B-tree of group nodes, symbol
// table nodes, a local heap of names), and one version-1 object header per dataset with
// dataspace, datatype, fill-value and contiguous data-layout messages.
//
// Writer layout (all addresses relative to byte 0, every object 8-byte aligned):
//   superblock | root object header | local heap header + names | B-tree node | symbol table
//   nodes | dataset object headers | raw data of each dataset
// The B-tree node and the symbol table nodes are allocated at their full size (2K entries) as the
// library reads them that way; the heap's free list is empty (head = 1, the library's end-of-list
// value); entries in a symbol table node are sorted by name.
#include <sys/stat.h>
#include <sys/types.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "afid_continua.h"
#include "afid_host_internal.h"
#include "afid_salinity.h"

namespace {

constexpr uint64_t kUndef = ~0ull;
constexpr uint8_t kSig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
constexpr int kLeafK = 4;          // symbol table node holds 2 * kLeafK entries
constexpr int kInternalK = 16;     // group B-tree node holds 2 * kInternalK children
constexpr size_t kEntrySize = 40;  // symbol table entry with 8-byte offsets
constexpr size_t kSnodSize = 8 + 2 * kLeafK * kEntrySize;
constexpr size_t kBtreeSize = 24 + (2 * kInternalK + 1) * 8 + 2 * kInternalK * 8;

size_t pad8(size_t n) { return (n + 7) & ~size_t(7); }

struct Out {
  std::vector<uint8_t> b;
  explicit Out(size_t n) : b(n, 0) {}
  void put(size_t pos, uint64_t v, int bytes) {
    for (int i = 0; i < bytes; ++i) b[pos + i] = (uint8_t)(v >> (8 * i));
  }
};

// Object header version 1 with the given messages (type, body); returns its bytes.
std::vector<uint8_t> object_header_v1(const std::vector<std::pair<int, std::vector<uint8_t>>> &msgs) {
  size_t body = 0;
  for (auto &m : msgs) body += 8 + pad8(m.second.size());
  std::vector<uint8_t> h(16 + body, 0);
  h[0] = 1;                                  // version
  h[2] = (uint8_t)msgs.size();               // number of messages (2 bytes)
  h[3] = (uint8_t)(msgs.size() >> 8);
  h[4] = 1;                                  // reference count (4 bytes)
  for (int i = 0; i < 4; ++i) h[8 + i] = (uint8_t)(body >> (8 * i));
  size_t p = 16;
  for (auto &m : msgs) {
    const size_t sz = pad8(m.second.size());
    h[p] = (uint8_t)m.first;
    h[p + 1] = (uint8_t)(m.first >> 8);
    h[p + 2] = (uint8_t)sz;
    h[p + 3] = (uint8_t)(sz >> 8);
    h[p + 4] = (m.first == 0x03 || m.first == 0x11) ? 1 : 0;  // datatype / symbol table: constant
    std::memcpy(&h[p + 8], m.second.data(), m.second.size());
    p += 8 + sz;
  }
  return h;
}

std::vector<uint8_t> le_bytes(std::initializer_list<std::pair<uint64_t, int>> fields) {
  std::vector<uint8_t> v;
  for (auto &f : fields)
    for (int i = 0; i < f.second; ++i) v.push_back((uint8_t)(f.first >> (8 * i)));
  return v;
}

std::vector<uint8_t> dataspace_msg(const afid_h5_dataset_t &d) {
  std::vector<uint8_t> v = {1, (uint8_t)d.rank, 0, 0, 0, 0, 0, 0};  // version 1, no max dims
  for (int r = 0; r < d.rank; ++r)
    for (int i = 0; i < 8; ++i) v.push_back((uint8_t)((uint64_t)d.dims[r] >> (8 * i)));
  return v;
}

std::vector<uint8_t> datatype_msg(int dtype) {
  if (dtype == AFID_H5_F64)
    // class 1 (floating point) version 1; little-endian, implied-MSB mantissa, sign bit 63;
    // 8 bytes; offset 0, precision 64, exponent at 52 of 11 bits, mantissa at 0 of 52, bias 1023
    return le_bytes({{0x11, 1}, {0x20, 1}, {63, 1}, {0, 1}, {8, 4}, {0, 2}, {64, 2}, {52, 1}, {11, 1},
                     {0, 1}, {52, 1}, {1023, 4}});
  // class 0 (fixed point) version 1; little-endian, signed; 4 bytes; offset 0, precision 32
  return le_bytes({{0x10, 1}, {0x08, 1}, {0, 1}, {0, 1}, {4, 4}, {0, 2}, {32, 2}});
}

size_t elem_size(int dtype) { return dtype == AFID_H5_F64 ? 8 : 4; }

int64_t elem_count(const afid_h5_dataset_t &d) {
  int64_t n = 1;
  for (int r = 0; r < d.rank; ++r) n *= d.dims[r];
  return n;
}

bool write_all(FILE *f, const void *p, size_t n) { return n == 0 || std::fwrite(p, 1, n, f) == n; }

}  // namespace

namespace {

// A group of the file being written: its members (sorted by name as C strcmp orders them) are
// datasets (ds >= 0, index into the caller's array) or groups (ds < 0).
struct GroupNode {
  std::vector<std::pair<std::string, int>> members;  // name, dataset index or -1 - child group
  std::vector<GroupNode> groups;
  // layout
  size_t a_oh = 0, a_heap = 0, a_heapdata = 0, heap_size = 0, a_snod = 0, nsnod = 0;
  std::vector<uint64_t> name_off;                     // per member
  std::vector<std::vector<size_t>> level_addr;        // B-tree node addresses per level (0 = leaves)
  size_t a_btree_root = 0;
};

// Insert dataset `ds` (or, with ds < 0, a group) under its '/'-separated path, creating the
// groups on the way; false on an empty component or a clash.
bool insert_path(GroupNode &g, const char *path, int ds) {
  const char *slash = std::strchr(path, '/');
  const std::string head = slash ? std::string(path, slash - path) : std::string(path);
  if (head.empty() || head.size() > 255) return false;
  for (auto &m : g.members)
    if (m.first == head) {
      if (m.second >= 0) return false;           // a dataset used again, or used as a group
      if (!slash) return ds < 0;                 // the group exists already: fine for a group entry
      return insert_path(g.groups[(size_t)(-1 - m.second)], slash + 1, ds);
    }
  if (!slash && ds >= 0) {
    g.members.emplace_back(head, ds);
    return true;
  }
  g.groups.emplace_back();
  g.members.emplace_back(head, -(int)g.groups.size());
  return slash ? insert_path(g.groups.back(), slash + 1, ds) : true;
}

void sort_members(GroupNode &g) {
  std::sort(g.members.begin(), g.members.end(), [](const std::pair<std::string, int> &a,
                                                   const std::pair<std::string, int> &b) {
    return std::strcmp(a.first.c_str(), b.first.c_str()) < 0;
  });
  for (auto &c : g.groups) sort_members(c);
}

// Addresses of a group's own structures: object header (symbol table message), local heap,
// B-tree nodes (root first, then the lower levels), symbol table nodes; then its child groups.
void place_group(GroupNode &g, size_t &a) {
  const size_t n = g.members.size();
  g.name_off.assign(n, 0);
  size_t heap = 8;
  for (size_t i = 0; i < n; ++i) {
    g.name_off[i] = heap;
    heap += pad8(g.members[i].first.size() + 1);
  }
  g.heap_size = heap;
  g.nsnod = (n + 2 * kLeafK - 1) / (2 * kLeafK);
  // B-tree levels: leaves over the symbol table nodes, each node up to 2K children
  std::vector<size_t> count{std::max<size_t>(1, (g.nsnod + 2 * kInternalK - 1) / (2 * kInternalK))};
  while (count.back() > 1) count.push_back((count.back() + 2 * kInternalK - 1) / (2 * kInternalK));
  g.a_oh = a;
  a += 16 + 8 + 16;
  g.a_heap = a;
  g.a_heapdata = a + 32;
  a += 32 + heap;
  g.level_addr.assign(count.size(), {});
  for (size_t lev = count.size(); lev-- > 0;)
    for (size_t c = 0; c < count[lev]; ++c) {
      g.level_addr[lev].push_back(a);
      a += kBtreeSize;
    }
  g.a_btree_root = g.level_addr.back()[0];
  g.a_snod = a;
  a += g.nsnod * kSnodSize;
  for (auto &c : g.groups) place_group(c, a);
}

// Serialise a placed group into the image `m` (dataset object header addresses in a_ds).
void emit_group(const GroupNode &g, Out &m, const std::vector<size_t> &a_ds) {
  const size_t n = g.members.size();
  {
    auto h = object_header_v1({{0x11, le_bytes({{g.a_btree_root, 8}, {g.a_heap, 8}})}});
    std::memcpy(&m.b[g.a_oh], h.data(), h.size());
  }
  std::memcpy(&m.b[g.a_heap], "HEAP", 4);
  m.put(g.a_heap + 8, g.heap_size, 8);
  m.put(g.a_heap + 16, 1, 8);  // empty free list
  m.put(g.a_heap + 24, g.a_heapdata, 8);
  for (size_t i = 0; i < n; ++i)
    std::memcpy(&m.b[g.a_heapdata + g.name_off[i]], g.members[i].first.data(), g.members[i].first.size());
  // symbol table nodes
  for (size_t c = 0; c < g.nsnod; ++c) {
    const size_t s = g.a_snod + c * kSnodSize, lo = c * 2 * kLeafK, hi = std::min(n, lo + 2 * kLeafK);
    std::memcpy(&m.b[s], "SNOD", 4);
    m.put(s + 4, 1, 1);
    m.put(s + 6, hi - lo, 2);
    for (size_t e = lo; e < hi; ++e) {
      const size_t p = s + 8 + (e - lo) * kEntrySize;
      const int id = g.members[e].second;
      m.put(p, g.name_off[e], 8);
      m.put(p + 8, id >= 0 ? a_ds[(size_t)id] : g.groups[(size_t)(-1 - id)].a_oh, 8);
    }
  }
  // B-tree nodes: children of a leaf are symbol table nodes, of a level-l node the level l-1
  // nodes; key 0 is the empty name, key c+1 the largest name under child c
  std::vector<uint64_t> child_addr(g.nsnod), child_key(g.nsnod);
  for (size_t c = 0; c < g.nsnod; ++c) {
    child_addr[c] = g.a_snod + c * kSnodSize;
    child_key[c] = g.name_off[std::min(n, (c + 1) * 2 * kLeafK) - 1];
  }
  for (size_t lev = 0; lev < g.level_addr.size(); ++lev) {
    const auto &nodes = g.level_addr[lev];
    std::vector<uint64_t> next_addr, next_key;
    for (size_t k = 0; k < nodes.size(); ++k) {
      const size_t b = nodes[k];
      const size_t lo = k * 2 * kInternalK, hi = std::min(child_addr.size(), lo + 2 * kInternalK);
      std::memcpy(&m.b[b], "TREE", 4);
      m.put(b + 4, 0, 1);
      m.put(b + 5, lev, 1);
      m.put(b + 6, hi - lo, 2);
      m.put(b + 8, k > 0 ? nodes[k - 1] : kUndef, 8);
      m.put(b + 16, k + 1 < nodes.size() ? nodes[k + 1] : kUndef, 8);
      size_t q = b + 24;
      m.put(q, 0, 8);
      q += 8;
      for (size_t c = lo; c < hi; ++c) {
        m.put(q, child_addr[c], 8);
        m.put(q + 8, child_key[c], 8);
        q += 16;
      }
      next_addr.push_back(b);
      next_key.push_back(hi > lo ? child_key[hi - 1] : 0);
    }
    child_addr.swap(next_addr);
    child_key.swap(next_key);
  }
  for (auto &c : g.groups) emit_group(c, m, a_ds);
}

}  // namespace

extern "C" int afid_h5_write(const char *path, int n, const afid_h5_dataset_t *sets) {
  return afid_guard([&]() -> int {
    if (!path || n < 0 || (n > 0 && !sets)) return AFID_E_INVALID;
    GroupNode root;
    for (int i = 0; i < n; ++i) {
      const afid_h5_dataset_t &d = sets[i];
      if (!d.name || !d.name[0] || std::strlen(d.name) > 4095) return AFID_E_INVALID;
      if (d.dtype == AFID_H5_GROUP) {
        if (!insert_path(root, d.name, -1)) return AFID_E_INVALID;
        continue;
      }
      if (d.rank < 1 || d.rank > AFID_H5_MAX_RANK || (d.dtype != AFID_H5_F64 && d.dtype != AFID_H5_I32))
        return AFID_E_INVALID;
      for (int r = 0; r < d.rank; ++r)
        if (d.dims[r] < 0) return AFID_E_INVALID;
      if (elem_count(d) > 0 && !d.data) return AFID_E_INVALID;
      if (!insert_path(root, d.name, i)) return AFID_E_INVALID;
    }
    sort_members(root);
    size_t a = 96;  // superblock
    place_group(root, a);
    const size_t meta_end = a;
    std::vector<size_t> a_ds(n), a_raw(n);
    std::vector<std::vector<uint8_t>> oh(n);
    auto is_ds = [&](int i) { return sets[i].dtype != AFID_H5_GROUP; };
    for (int i = 0; i < n; ++i) {  // headers first (their size does not depend on the raw address)
      if (!is_ds(i)) continue;
      oh[i] = object_header_v1({{0x01, dataspace_msg(sets[i])},
                                {0x03, datatype_msg(sets[i].dtype)},
                                {0x05, {2, 2, 2, 1, 0, 0, 0, 0}},  // fill value v2: late, if set, defined, size 0
                                {0x08, std::vector<uint8_t>(18, 0)}});
      a_ds[i] = a;
      a += oh[i].size();
    }
    for (int i = 0; i < n; ++i) {
      if (!is_ds(i)) continue;
      a_raw[i] = a;
      a += pad8((size_t)elem_count(sets[i]) * elem_size(sets[i].dtype));
    }
    const size_t eof = a;
    for (int i = 0; i < n; ++i) {  // the layout message: version 3, contiguous, address, size
      if (!is_ds(i)) continue;
      const size_t lay = 16 + (8 + pad8(dataspace_msg(sets[i]).size())) +
                         (8 + pad8(datatype_msg(sets[i].dtype).size())) + (8 + 8) + 8;
      const uint64_t bytes = (uint64_t)elem_count(sets[i]) * elem_size(sets[i].dtype);
      oh[i][lay] = 3;
      oh[i][lay + 1] = 1;
      for (int k = 0; k < 8; ++k) {
        oh[i][lay + 2 + k] = (uint8_t)((uint64_t)a_raw[i] >> (8 * k));
        oh[i][lay + 10 + k] = (uint8_t)(bytes >> (8 * k));
      }
    }

    Out m(meta_end);
    // superblock version 0
    std::memcpy(&m.b[0], kSig, 8);
    m.put(13, 8, 1);  // size of offsets
    m.put(14, 8, 1);  // size of lengths
    m.put(16, kLeafK, 2);
    m.put(18, kInternalK, 2);
    m.put(24, 0, 8);        // base address
    m.put(32, kUndef, 8);   // free-space info
    m.put(40, eof, 8);      // end of file
    m.put(48, kUndef, 8);   // driver info
    m.put(56, 0, 8);        // root entry: link name offset
    m.put(64, root.a_oh, 8);  //   object header address
    m.put(72, 1, 4);        //   cache type 1: scratch holds B-tree and heap addresses
    m.put(80, root.a_btree_root, 8);
    m.put(88, root.a_heap, 8);
    emit_group(root, m, a_ds);

    FILE *f = std::fopen(path, "wb");
    if (!f) return AFID_E_IO;
    bool ok = write_all(f, m.b.data(), m.b.size());
    for (int i = 0; i < n && ok; ++i) ok = write_all(f, oh[i].data(), oh[i].size());
    static const uint8_t zeros[8] = {0};
    for (int i = 0; i < n && ok; ++i) {
      if (!is_ds(i)) continue;
      const size_t bytes = (size_t)elem_count(sets[i]) * elem_size(sets[i].dtype);
      ok = write_all(f, sets[i].data, bytes) && write_all(f, zeros, pad8(bytes) - bytes);
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? AFID_OK : AFID_E_IO;
  });
}

// ---- reader --------------------------------------------------------------------------------
namespace {

struct Msg {
  int type;
  std::vector<uint8_t> body;
};

struct DsInfo {
  int rank = -1;
  int64_t dims[AFID_H5_MAX_RANK] = {0, 0, 0, 0};
  int cls = -1;          // 0 fixed point, 1 floating point
  int size = 0;          // bytes per element
  bool big_endian = false, is_signed = true;
  bool compact = false, allocated = false;
  uint64_t addr = 0;
  std::vector<uint8_t> inline_data;
};

uint64_t le(const uint8_t *p, int n) {
  uint64_t v = 0;
  for (int i = 0; i < n; ++i) v |= (uint64_t)p[i] << (8 * i);
  return v;
}

class Reader {
 public:
  ~Reader() {
    if (f_) std::fclose(f_);
  }
  bool open(const char *path) {
    f_ = std::fopen(path, "rb");
    if (!f_) return false;
    if (std::fseek(f_, 0, SEEK_END) != 0) return false;
    const long end = std::ftell(f_);
    if (end < 0) return false;
    fsize_ = (uint64_t)end;
    for (uint64_t pos = 0; pos + 8 <= fsize_; pos = pos ? pos * 2 : 512) {
      uint8_t s[8];
      if (!raw(pos, s, 8)) return false;
      if (std::memcmp(s, kSig, 8) == 0) return superblock(pos);
    }
    return false;
  }

  // Object header of the '/'-separated path below the root group.
  bool find(const char *name, uint64_t *hdr) {
    uint64_t cur = root_;
    const char *p = name;
    for (int depth = 0; depth < 32; ++depth) {
      const char *slash = std::strchr(p, '/');
      const std::string comp = slash ? std::string(p, slash - p) : std::string(p);
      if (comp.empty() || !lookup(cur, comp.c_str(), &cur, 0)) return false;
      if (!slash) {
        *hdr = cur;
        return true;
      }
      p = slash + 1;
    }
    return false;
  }

  bool dataset(uint64_t hdr, DsInfo &d) {
    std::vector<Msg> msgs;
    if (!messages(hdr, msgs)) return false;
    bool have_space = false, have_type = false, have_layout = false;
    for (auto &m : msgs) {
      const uint8_t *b = m.body.data();
      const size_t n = m.body.size();
      if (m.type == 0x01) {  // dataspace
        if (n < 4) return false;
        const int version = b[0], rank = b[1];
        size_t r;
        if (version == 1) r = 8;
        else if (version == 2) {
          r = 4;
          if (b[3] == 0) { d.rank = 0; have_space = true; continue; }  // scalar
          if (b[3] != 1) return false;                                  // null dataspace
        } else return false;
        if (rank > AFID_H5_MAX_RANK || n < r + (size_t)rank * sl_) return false;
        d.rank = rank;
        for (int i = 0; i < rank; ++i) d.dims[i] = (int64_t)le(b + r + i * sl_, sl_);
        have_space = true;
      } else if (m.type == 0x03) {  // datatype
        if (n < 8) return false;
        d.cls = b[0] & 0x0f;
        d.big_endian = b[1] & 1;
        d.is_signed = (b[1] & 0x08) != 0;
        d.size = (int)le(b + 4, 4);
        if (d.cls == 1 && d.size != 4 && d.size != 8) return false;
        if (d.cls == 0 && d.size != 1 && d.size != 2 && d.size != 4 && d.size != 8) return false;
        if (d.cls != 0 && d.cls != 1) return false;
        have_type = true;
      } else if (m.type == 0x08) {  // data layout
        if (n < 2) return false;
        const int version = b[0];
        if (version == 3 || version == 4) {
          const int cls = b[1];
          if (cls == 0) {
            const size_t len = (size_t)le(b + 2, 2);
            if (n < 4 + len) return false;
            d.compact = true;
            d.inline_data.assign(b + 4, b + 4 + len);
          } else if (cls == 1) {
            if (n < 2 + (size_t)so_ + sl_) return false;
            d.addr = le(b + 2, so_);
          } else return false;  // chunked or virtual
        } else if (version == 1 || version == 2) {
          if (n < 8) return false;
          const int rank = b[1], cls = b[2];
          if (cls == 1) {
            if (n < 8 + (size_t)so_) return false;
            d.addr = le(b + 8, so_);
          } else if (cls == 0) {
            const size_t r = 8 + 4 * (size_t)rank;
            if (n < r + 4) return false;
            const size_t len = (size_t)le(b + r, 4);
            if (n < r + 4 + len) return false;
            d.compact = true;
            d.inline_data.assign(b + r + 4, b + r + 4 + len);
          } else return false;
        } else return false;
        have_layout = true;
      } else if (m.type == 0x0b) {
        return false;  // filter pipeline
      }
    }
    d.allocated = d.compact || (d.addr != undef_addr());
    if (!(have_space && have_type && have_layout)) return false;
    // the shape must be non-negative, its element count must not overflow, and the data must
    // lie inside the file (or inside the header, for compact storage)
    uint64_t count = 1;
    for (int i = 0; i < d.rank; ++i) {
      if (d.dims[i] < 0 || (uint64_t)d.dims[i] > (1ull << 40)) return false;
      if (d.dims[i] != 0 && count > (1ull << 48) / (uint64_t)d.dims[i]) return false;
      count *= (uint64_t)d.dims[i];
    }
    const uint64_t bytes = count * (uint64_t)d.size;
    if (d.compact) return bytes <= d.inline_data.size();
    if (d.allocated) return d.addr <= fsize_ && base_ <= fsize_ - d.addr && bytes <= fsize_ - base_ - d.addr;
    return true;
  }

  // Read count elements of dataset d converted to double.
  bool read_f64(const DsInfo &d, double *out, int64_t count) {
    const size_t es = (size_t)d.size;
    const uint16_t probe = 1;
    const bool host_le = *reinterpret_cast<const uint8_t *>(&probe) == 1;
    if (d.cls == 1 && es == 8 && !d.big_endian && host_le && d.allocated && !d.compact)
      return raw(base_ + d.addr, out, (size_t)count * 8);  // the on-disk bytes are the host's doubles
    const size_t chunk = 1 << 20;  // elements per pass
    std::vector<uint8_t> buf;
    for (int64_t i0 = 0; i0 < count; i0 += (int64_t)chunk) {
      const size_t m = (size_t)std::min<int64_t>((int64_t)chunk, count - i0);
      buf.resize(m * es);
      if (d.compact) {
        if ((i0 + (int64_t)m) * es > d.inline_data.size()) return false;
        std::memcpy(buf.data(), d.inline_data.data() + i0 * es, m * es);
      } else if (!d.allocated) {
        std::fill(buf.begin(), buf.end(), 0);  // never written: the default fill value is zero
      } else if (!raw(base_ + d.addr + (uint64_t)i0 * es, buf.data(), m * es)) {
        return false;
      }
      for (size_t k = 0; k < m; ++k) {
        uint8_t e[8];
        for (size_t j = 0; j < es; ++j) e[j] = d.big_endian ? buf[k * es + es - 1 - j] : buf[k * es + j];
        double v;
        if (d.cls == 1) {
          if (es == 8) std::memcpy(&v, e, 8);
          else {
            float x;
            std::memcpy(&x, e, 4);
            v = x;
          }
        } else {
          uint64_t u = le(e, (int)es);
          if (d.is_signed && es < 8 && (u >> (8 * es - 1)) & 1) u |= ~0ull << (8 * es);
          v = d.is_signed ? (double)(int64_t)u : (double)u;
        }
        out[i0 + (int64_t)k] = v;
      }
    }
    return true;
  }

 private:
  FILE *f_ = nullptr;
  uint64_t fsize_ = 0, base_ = 0, root_ = 0;
  // B-tree and symbol-table nodes one lookup may visit: a damaged tree whose nodes point back at
  // themselves would otherwise be walked an exponential number of times
  long long node_budget_ = 0;
  int so_ = 8, sl_ = 8;

  uint64_t undef_addr() const { return so_ == 8 ? kUndef : ((1ull << (8 * so_)) - 1); }

  bool raw(uint64_t pos, void *dst, size_t n) {
    if (pos > fsize_ || n > fsize_ - pos) return false;
    if (std::fseek(f_, (long)pos, SEEK_SET) != 0) return false;
    return std::fread(dst, 1, n, f_) == n;
  }
  bool at(uint64_t addr, std::vector<uint8_t> &v, size_t n) {
    v.resize(n);
    return raw(base_ + addr, v.data(), n);
  }

  bool superblock(uint64_t pos) {
    uint8_t s[256];
    const size_t n = (size_t)std::min<uint64_t>(sizeof(s), fsize_ - pos);
    if (n < 48 || !raw(pos, s, n)) return false;
    const int version = s[8];
    if (version == 0 || version == 1) {
      so_ = s[13];
      sl_ = s[14];
      if ((so_ != 4 && so_ != 8) || (sl_ != 4 && sl_ != 8)) return false;
      size_t q = 24 + (version == 1 ? 4 : 0);
      if (q + 4 * so_ + 2 * so_ > n) return false;
      base_ = le(s + q, so_);
      q += 4 * so_;                  // base, free space, end of file, driver block
      root_ = le(s + q + so_, so_);  // root entry: link name offset, object header address
    } else if (version == 2 || version == 3) {
      so_ = s[9];
      sl_ = s[10];
      if ((so_ != 4 && so_ != 8) || (sl_ != 4 && sl_ != 8)) return false;
      const size_t q = 12;
      if (q + 4 * so_ > n) return false;
      base_ = le(s + q, so_);
      root_ = le(s + q + 3 * so_, so_);  // base, extension, end of file, root object header
    } else {
      return false;
    }
    return true;
  }

  bool messages(uint64_t addr, std::vector<Msg> &out) {
    std::vector<uint8_t> h;
    if (!at(addr, h, 16)) return false;
    struct Chunk { uint64_t addr, len; bool v2_cont; };
    std::vector<Chunk> todo;
    if (std::memcmp(h.data(), "OHDR", 4) == 0) {
      const int flags = h[5];
      size_t q = 6 + ((flags & 0x20) ? 16 : 0) + ((flags & 0x10) ? 4 : 0);
      const int w = 1 << (flags & 3);
      std::vector<uint8_t> pre;
      if (!at(addr, pre, q + w)) return false;
      const uint64_t len = le(pre.data() + q, w);
      const bool order = flags & 0x04;
      todo.push_back({addr + q + w, len, false});
      for (size_t c = 0; c < todo.size() && c < 64; ++c) {
        std::vector<uint8_t> b;
        if (todo[c].len > (64u << 20) || !at(todo[c].addr, b, (size_t)todo[c].len)) return false;
        size_t r = 0, end = b.size();
        if (todo[c].v2_cont) {
          if (end < 8 || std::memcmp(b.data(), "OCHK", 4) != 0) return false;
          r = 4;
          end -= 4;
        }
        const size_t mh = order ? 6 : 4;
        while (r + mh <= end) {
          const int type = b[r];
          const size_t sz = (size_t)le(&b[r + 1], 2);
          r += mh;
          if (r + sz > end) break;  // gap at the end of the chunk
          if (type == 0x10) {
            if (sz < (size_t)so_ + sl_) return false;
            todo.push_back({le(&b[r], so_), le(&b[r + so_], sl_), true});
          } else {
            out.push_back({type, std::vector<uint8_t>(b.begin() + r, b.begin() + r + sz)});
          }
          r += sz;
        }
      }
      return true;
    }
    if (h[0] != 1) return false;
    const size_t nmsg = (size_t)le(&h[2], 2);
    todo.push_back({addr + 16, le(&h[8], 4), false});
    for (size_t c = 0; c < todo.size() && c < 64 && out.size() < nmsg; ++c) {
      std::vector<uint8_t> b;
      if (todo[c].len > (64u << 20) || !at(todo[c].addr, b, (size_t)todo[c].len)) return false;
      size_t r = 0;
      while (r + 8 <= b.size()) {
        const int type = (int)le(&b[r], 2);
        const size_t sz = (size_t)le(&b[r + 2], 2);
        r += 8;
        if (r + sz > b.size()) return false;
        if (type == 0x10) {
          if (sz < (size_t)so_ + sl_) return false;
          todo.push_back({le(&b[r], so_), le(&b[r + so_], sl_), false});
        } else {
          out.push_back({type, std::vector<uint8_t>(b.begin() + r, b.begin() + r + sz)});
        }
        r += sz;
      }
    }
    return true;
  }

  bool heap_name(uint64_t heap_data, uint64_t off, std::string &s) {
    s.clear();
    char c[64];
    for (uint64_t p = off;; p += sizeof(c)) {
      const size_t n = (size_t)std::min<uint64_t>(sizeof(c), fsize_ - std::min(fsize_, base_ + heap_data + p));
      if (n == 0 || !raw(base_ + heap_data + p, c, n)) return false;
      for (size_t i = 0; i < n; ++i) {
        if (c[i] == 0) return true;
        s.push_back(c[i]);
        if (s.size() > 4096) return false;
      }
    }
  }

  // Symbol table group: walk the B-tree of group nodes down to the symbol table nodes.
  bool btree_find(uint64_t node, uint64_t heap_data, const char *name, uint64_t *hdr, int depth) {
    if (depth > 16 || --node_budget_ < 0) return false;
    std::vector<uint8_t> b;
    if (!at(node, b, 8 + 2 * (size_t)so_)) return false;
    if (std::memcmp(b.data(), "TREE", 4) != 0 || b[4] != 0) return false;
    const int level = b[5];
    const size_t used = (size_t)le(&b[6], 2);
    const size_t body = 8 + 2 * (size_t)so_ + (used + 1) * sl_ + used * so_;
    if (used > 4096 || !at(node, b, body)) return false;
    size_t q = 8 + 2 * so_ + sl_;
    for (size_t i = 0; i < used; ++i, q += so_ + sl_) {
      const uint64_t child = le(&b[q], so_);
      if (level > 0) {
        if (btree_find(child, heap_data, name, hdr, depth + 1)) return true;
        continue;
      }
      std::vector<uint8_t> s;
      if (!at(child, s, 8)) return false;
      if (std::memcmp(s.data(), "SNOD", 4) != 0) return false;
      const size_t nsym = (size_t)le(&s[6], 2), es = 2 * (size_t)so_ + 24;
      if (nsym > 4096 || (node_budget_ -= (long long)nsym + 1) < 0 || !at(child, s, 8 + nsym * es)) return false;
      for (size_t e = 0; e < nsym; ++e) {
        std::string nm;
        if (!heap_name(heap_data, le(&s[8 + e * es], so_), nm)) return false;
        if (nm == name) {
          *hdr = le(&s[8 + e * es + so_], so_);
          return true;
        }
      }
    }
    return false;
  }

  bool lookup(uint64_t group, const char *name, uint64_t *hdr, int depth) {
    std::vector<Msg> msgs;
    if (depth > 0 || !messages(group, msgs)) return false;
    for (auto &m : msgs) {
      const uint8_t *b = m.body.data();
      const size_t n = m.body.size();
      if (m.type == 0x11) {  // symbol table: B-tree and local heap
        if (n < 2 * (size_t)so_) return false;
        const uint64_t btree = le(b, so_), heap = le(b + so_, so_);
        std::vector<uint8_t> hh;
        if (!at(heap, hh, 8 + 2 * (size_t)sl_ + so_) || std::memcmp(hh.data(), "HEAP", 4) != 0) return false;
        const uint64_t heap_data = le(&hh[8 + 2 * sl_], so_);
        node_budget_ = 1 << 20;
        return btree_find(btree, heap_data, name, hdr, 0);
      }
      if (m.type == 0x06) {  // link message (compact storage)
        if (n < 2) continue;
        const int flags = b[1];
        size_t r = 2;
        int ltype = 0;
        if (flags & 0x08) ltype = b[r++];
        if (flags & 0x04) r += 8;
        if (flags & 0x10) r += 1;
        const int w = 1 << (flags & 3);
        if (r + w > n) continue;
        const size_t len = (size_t)le(b + r, w);
        r += w;
        if (r + len + so_ > n) continue;
        if (ltype == 0 && len == std::strlen(name) && std::memcmp(b + r, name, len) == 0) {
          *hdr = le(b + r + len, so_);
          return true;
        }
      }
    }
    return false;
  }
};

int open_dataset(const char *path, const char *name, Reader &rd, DsInfo &d) {
  if (!path || !name) return AFID_E_INVALID;
  uint64_t hdr = 0;
  if (!rd.open(path) || !rd.find(name, &hdr) || !rd.dataset(hdr, d)) return AFID_E_IO;
  return AFID_OK;
}

}  // namespace

extern "C" int afid_h5_info(const char *path, const char *name, int *dtype, int *rank,
                            int64_t dims[AFID_H5_MAX_RANK]) {
  return afid_guard([&]() -> int {
    Reader rd;
    DsInfo d;
    const int s = open_dataset(path, name, rd, d);
    if (s != AFID_OK) return s;
    if (dtype) *dtype = d.cls == 1 ? AFID_H5_F64 : AFID_H5_I32;
    if (rank) *rank = d.rank;
    if (dims)
      for (int i = 0; i < AFID_H5_MAX_RANK; ++i) dims[i] = i < d.rank ? d.dims[i] : 0;
    return AFID_OK;
  });
}

extern "C" int afid_h5_read_f64(const char *path, const char *name, double *out, int64_t count) {
  return afid_guard([&]() -> int {
    if (!out || count < 0) return AFID_E_INVALID;
    Reader rd;
    DsInfo d;
    const int s = open_dataset(path, name, rd, d);
    if (s != AFID_OK) return s;
    int64_t n = 1;
    for (int i = 0; i < d.rank; ++i) n *= d.dims[i];
    if (n != count) return AFID_E_INVALID;
    return rd.read_f64(d, out, count) ? AFID_OK : AFID_E_IO;
  });
}

// ---- continua files --------------------------------------------------------------------------
namespace {

bool ensure_dir(const std::string &d) {
  struct stat st;
  if (stat(d.c_str(), &st) == 0) return S_ISDIR(st.st_mode);
  return mkdir(d.c_str(), 0755) == 0 || errno == EEXIST;
}

bool file_exists(const std::string &p) {
  struct stat st;
  return stat(p.c_str(), &st) == 0 && S_ISREG(st.st_mode);
}

// One field file: dataset "var" with C-order dims (n3, n2, n1), from a packed host array whose x
// extent is src_x (<= n1; the remaining x nodes are written as zero).
int write_field(const std::string &path, const double *src, int src_x, int n1, int n2, int n3) {
  const double *data = src;
  std::vector<double> padded;
  if (src_x != n1) {
    padded.assign((size_t)n1 * n2 * n3, 0.0);
    for (size_t c = 0; c < (size_t)n2 * n3; ++c)
      std::memcpy(&padded[c * n1], src + c * src_x, sizeof(double) * src_x);
    data = padded.data();
  }
  afid_h5_dataset_t d{};
  d.name = "var";
  d.dtype = AFID_H5_F64;
  d.rank = 3;
  d.dims[0] = n3;
  d.dims[1] = n2;
  d.dims[2] = n1;
  d.data = data;
  return afid_h5_write(path.c_str(), 1, &d);
}

// Read dataset "var" with C-order dims (n3, n2, n1) into a packed array of x extent dst_x <= n1.
int read_field(const std::string &path, double *dst, int dst_x, int n1, int n2, int n3) {
  int dtype = 0, rank = 0;
  int64_t dims[AFID_H5_MAX_RANK];
  int s = afid_h5_info(path.c_str(), "var", &dtype, &rank, dims);
  if (s != AFID_OK) return s;
  if (rank != 3 || dims[0] != n3 || dims[1] != n2 || dims[2] != n1) return AFID_E_INVALID;
  const int64_t count = (int64_t)n1 * n2 * n3;
  if (dst_x == n1) return afid_h5_read_f64(path.c_str(), "var", dst, count);
  std::vector<double> full((size_t)count);
  if ((s = afid_h5_read_f64(path.c_str(), "var", full.data(), count)) != AFID_OK) return s;
  for (size_t c = 0; c < (size_t)n2 * n3; ++c) std::memcpy(dst + c * dst_x, &full[c * n1], sizeof(double) * dst_x);
  return AFID_OK;
}

int read_scalar(const std::string &path, const char *name, double *v) {
  int dtype = 0, rank = 0;
  int64_t dims[AFID_H5_MAX_RANK];
  int s = afid_h5_info(path.c_str(), name, &dtype, &rank, dims);
  if (s != AFID_OK) return s;
  int64_t n = 1;
  for (int i = 0; i < rank; ++i) n *= dims[i];
  if (n != 1) return AFID_E_IO;
  return afid_h5_read_f64(path.c_str(), name, v, 1);
}

}  // namespace

extern "C" int afid_continua_master_from_input(const afid_input_t *in, double time, afid_continua_master_t *m) {
  return afid_guard([&]() -> int {
    if (!in || !m) return AFID_E_INVALID;
    *m = afid_continua_master_t{};
    m->nx = in->nxm + 1;
    m->ny = in->nym + 1;
    m->nz = in->nzm + 1;
    m->ylen = in->ylen;
    m->zlen = in->zlen;
    m->time = time;
    m->istr3 = in->istr3;
    m->str3 = in->str3;
    m->multires = in->multires ? 1 : 0;
    if (m->multires) {
      m->nxr = in->nxmr + 1;
      m->nyr = in->nymr + 1;
      m->nzr = in->nzmr + 1;
      m->istr3r = in->istr3r;
    }
    return AFID_OK;
  });
}

extern "C" int afid_write_flow_field(const char *dir, int final, double save_3d, const afid_continua_master_t *m,
                                     const double *vx, const double *vy, const double *vz, const double *temp,
                                     const double *pr, const double *sal) {
  return afid_guard([&]() -> int {
    if (!dir || !m || !vx || !vy || !vz || !temp || (final && !pr)) return AFID_E_INVALID;
    const int nx = m->nx, nym = m->ny - 1, nzm = m->nz - 1;
    if (nx < 2 || nym < 1 || nzm < 1) return AFID_E_INVALID;
    const bool with_sal = m->multires && sal;
    if (with_sal && (m->nxr < 2 || m->nyr < 2 || m->nzr < 2)) return AFID_E_INVALID;
    std::string base = dir;
    if (!ensure_dir(base)) return AFID_E_IO;
    if (final) {
      base += "/continua";
    } else {  // WriteFlowField.F90:22-26: frame = nint(time / save_3D), written as i5.5
      if (!(save_3d > 0.0)) return AFID_E_INVALID;
      const double fr = std::round(m->time / save_3d);  // nint: halves away from zero
      if (!(fr >= 0.0 && fr <= 99999.0)) return AFID_E_INVALID;
      char frame[8];
      std::snprintf(frame, sizeof(frame), "%05d", (int)fr);
      base += "/fields";
      if (!ensure_dir(base)) return AFID_E_IO;
      base += std::string("/") + frame;
    }
    int s;
    if ((s = write_field(base + "_temp.h5", temp, nx, nx, nym, nzm)) != AFID_OK) return s;
    if ((s = write_field(base + "_vx.h5", vx, nx, nx, nym, nzm)) != AFID_OK) return s;
    if ((s = write_field(base + "_vy.h5", vy, nx, nx, nym, nzm)) != AFID_OK) return s;
    if ((s = write_field(base + "_vz.h5", vz, nx, nx, nym, nzm)) != AFID_OK) return s;
    if (with_sal && (s = write_field(base + "_sal.h5", sal, m->nxr - 1, m->nxr, m->nyr - 1, m->nzr - 1)) != AFID_OK)
      return s;
    if (!final) return AFID_OK;
    if ((s = write_field(base + "_pr.h5", pr, nx, nx, nym, nzm)) != AFID_OK) return s;
    // continua_master.h5 (WriteFlowField.F90:51-82): one-element datasets
    const int32_t ints[7] = {m->nx, m->ny, m->nz, m->istr3, m->nxr, m->nyr, m->nzr};
    const int32_t istr3r = m->istr3r;
    const double reals[4] = {m->ylen, m->zlen, m->time, m->str3};
    afid_h5_dataset_t d[12];
    int n = 0;
    auto add = [&](const char *name, int dtype, const void *p) {
      d[n] = afid_h5_dataset_t{};
      d[n].name = name;
      d[n].dtype = dtype;
      d[n].rank = 1;
      d[n].dims[0] = 1;
      d[n].data = p;
      ++n;
    };
    add("nx", AFID_H5_I32, &ints[0]);
    add("ny", AFID_H5_I32, &ints[1]);
    add("nz", AFID_H5_I32, &ints[2]);
    add("ylen", AFID_H5_F64, &reals[0]);
    add("zlen", AFID_H5_F64, &reals[1]);
    add("time", AFID_H5_F64, &reals[2]);
    add("istr3", AFID_H5_I32, &ints[3]);
    add("str3", AFID_H5_F64, &reals[3]);
    if (m->multires) {
      add("nxr", AFID_H5_I32, &ints[4]);
      add("nyr", AFID_H5_I32, &ints[5]);
      add("nzr", AFID_H5_I32, &ints[6]);
      add("istr3r", AFID_H5_I32, &istr3r);
    }
    return afid_h5_write((std::string(dir) + "/continua_master.h5").c_str(), n, d);
  });
}

extern "C" int afid_read_continua_master(const char *dir, int multires, afid_continua_master_t *m) {
  return afid_guard([&]() -> int {
    if (!dir || !m) return AFID_E_INVALID;
    const std::string p = std::string(dir) + "/continua_master.h5";
    if (!file_exists(p)) return AFID_E_IO;  // "Continuation files not found" (ReadFlowInterp.F90:25-29)
    afid_continua_master_t r{};
    double v[12];
    const char *names[12] = {"nx", "ny", "nz", "time", "istr3", "str3", "ylen", "zlen", "nxr", "nyr", "nzr", "istr3r"};
    const int count = multires ? 12 : 8;
    for (int i = 0; i < count; ++i) {
      const int s = read_scalar(p, names[i], &v[i]);
      if (s != AFID_OK) return s;
    }
    r.nx = (int)v[0];
    r.ny = (int)v[1];
    r.nz = (int)v[2];
    r.time = v[3];
    r.istr3 = (int)v[4];
    r.str3 = v[5];
    r.ylen = v[6];
    r.zlen = v[7];
    r.multires = multires ? 1 : 0;
    if (multires) {
      r.nxr = (int)v[8];
      r.nyr = (int)v[9];
      r.nzr = (int)v[10];
      r.istr3r = (int)v[11];
    }
    *m = r;
    return AFID_OK;
  });
}

extern "C" int afid_read_flow_field(const char *dir, const afid_continua_master_t *cur, double *time_out, double *vx,
                                    double *vy, double *vz, double *temp, double *pr, int *pr_read, double *sal) {
  return afid_guard([&]() -> int {
    if (!dir || !cur || !vx || !vy || !vz || !temp) return AFID_E_INVALID;
    afid_continua_master_t old{};
    int s = afid_read_continua_master(dir, cur->multires, &old);
    if (s != AFID_OK) return s;
    // ReadFlowInterp.F90:76-82: the domain size must match
    if (std::fabs(cur->ylen - old.ylen) > 1e-8 || std::fabs(cur->zlen - old.zlen) > 1e-8) return AFID_E_INVALID;
    // ReadFlowInterp.F90:85-89: a different grid needs the interpolating restart
    if (cur->nx != old.nx || cur->ny != old.ny || cur->nz != old.nz || cur->istr3 != old.istr3 ||
        std::fabs(cur->str3 - old.str3) > 1e-8 ||
        (cur->multires && (cur->nxr != old.nxr || cur->nyr != old.nyr || cur->nzr != old.nzr || cur->istr3r != old.istr3r)))
      return AFID_E_INVALID;
    const std::string base = std::string(dir) + "/continua";
    const int nx = cur->nx, nym = cur->ny - 1, nzm = cur->nz - 1;
    if ((s = read_field(base + "_vx.h5", vx, nx, nx, nym, nzm)) != AFID_OK) return s;
    if ((s = read_field(base + "_vy.h5", vy, nx, nx, nym, nzm)) != AFID_OK) return s;
    if ((s = read_field(base + "_vz.h5", vz, nx, nx, nym, nzm)) != AFID_OK) return s;
    if ((s = read_field(base + "_temp.h5", temp, nx, nx, nym, nzm)) != AFID_OK) return s;
    if (cur->multires && sal &&
        (s = read_field(base + "_sal.h5", sal, cur->nxr - 1, cur->nxr, cur->nyr - 1, cur->nzr - 1)) != AFID_OK)
      return s;
    int got_pr = 0;
    if (pr && file_exists(base + "_pr.h5")) {  // ReadFlowInterp.F90:157-162
      if ((s = read_field(base + "_pr.h5", pr, nx, nx, nym, nzm)) != AFID_OK) return s;
      got_pr = 1;
    }
    if (pr_read) *pr_read = got_pr;
    if (time_out) *time_out = old.time;
    return AFID_OK;
  });
}

extern "C" int afid_gpu_write_flow_field(afid_ctx_t *ctx, const char *dir, int final, double save_3d,
                                         const afid_continua_master_t *m) {
  return afid_guard([&]() -> int {
    if (!ctx || !dir || !m) return AFID_E_INVALID;
    int dims[6];
    int s = afid_gpu_dims(ctx, dims);
    if (s != AFID_OK) return s;
    if (m->nx != dims[0] + 1 || m->ny != dims[1] + 1 || m->nz != dims[2] + 1) return AFID_E_INVALID;
    const bool with_sal = m->multires && dims[3] > 0;
    if (with_sal && (m->nxr != dims[3] + 1 || m->nyr != dims[4] + 1 || m->nzr != dims[5] + 1)) return AFID_E_INVALID;
    const int nx = m->nx, nym = dims[1], nzm = dims[2];
    const size_t n = (size_t)nx * nym * nzm;
    std::vector<double> f(5 * n);
    double *vx = f.data(), *vy = vx + n, *vz = vy + n, *temp = vz + n, *pr = temp + n;
    if ((s = afid_gpu_download(ctx, vx, vy, vz, temp, pr, nx, nym)) != AFID_OK) return s;
    std::vector<double> sal;
    if (with_sal) {
      sal.resize((size_t)dims[3] * dims[4] * dims[5]);
      if ((s = afid_gpu_sal_download(ctx, sal.data(), dims[3], dims[4])) != AFID_OK) return s;
    }
    return afid_write_flow_field(dir, final, save_3d, m, vx, vy, vz, temp, pr, with_sal ? sal.data() : nullptr);
  });
}

// WriteSpectra (spectra.F90:169-196): the time-averaged power spectra of vx, vy, vz and temp as
// <dir>/{vx,vy,vz,te}_spectrum.h5 (afid_gpu_spectra_read gives each divided by the averaging
// interval, as the reference divides by time - tav_start).
extern "C" int afid_gpu_write_spectra(afid_ctx_t *ctx, const char *dir) {
  return afid_guard([&]() -> int {
    static const char *const kFile[4] = {"vx_spectrum.h5", "vy_spectrum.h5", "vz_spectrum.h5", "te_spectrum.h5"};
    if (!ctx || !dir) return AFID_E_INVALID;
    int dims[6];
    int s = afid_gpu_dims(ctx, dims);
    if (s != AFID_OK) return s;
    const int nxm = dims[0], nym = dims[1], nzm = dims[2];
    if (!ensure_dir(dir)) return AFID_E_IO;
    std::vector<double> half((size_t)nxm * (nym / 2 + 1) * nzm);
    for (int w = 0; w < 4; ++w) {
      double tav = 0.0;
      if ((s = afid_gpu_spectra_read(ctx, w, half.data(), &tav)) != AFID_OK) return s;
      if ((s = afid_write_spectrum((std::string(dir) + "/" + kFile[w]).c_str(), nxm, nym, nzm, half.data())) != AFID_OK)
        return s;
    }
    return AFID_OK;
  });
}

extern "C" int afid_gpu_read_flow_field(afid_ctx_t *ctx, const char *dir, const afid_continua_master_t *cur,
                                        double *time_out) {
  return afid_guard([&]() -> int {
    if (!ctx || !dir || !cur) return AFID_E_INVALID;
    int dims[6];
    int s = afid_gpu_dims(ctx, dims);
    if (s != AFID_OK) return s;
    if (cur->nx != dims[0] + 1 || cur->ny != dims[1] + 1 || cur->nz != dims[2] + 1) return AFID_E_INVALID;
    const bool with_sal = cur->multires && dims[3] > 0;
    if (with_sal && (cur->nxr != dims[3] + 1 || cur->nyr != dims[4] + 1 || cur->nzr != dims[5] + 1))
      return AFID_E_INVALID;
    const int nx = cur->nx, nym = dims[1], nzm = dims[2];
    const size_t n = (size_t)nx * nym * nzm;
    std::vector<double> f(5 * n, 0.0);
    double *vx = f.data(), *vy = vx + n, *vz = vy + n, *temp = vz + n, *pr = temp + n;
    std::vector<double> sal(with_sal ? (size_t)dims[3] * dims[4] * dims[5] : 0);
    int pr_read = 0;
    double t = 0.0;
    if ((s = afid_read_flow_field(dir, cur, &t, vx, vy, vz, temp, pr, &pr_read, with_sal ? sal.data() : nullptr)) !=
        AFID_OK)
      return s;
    if ((s = afid_gpu_upload(ctx, vx, vy, vz, temp, pr, nx, nym)) != AFID_OK) return s;
    if (with_sal && (s = afid_gpu_sal_upload(ctx, sal.data(), dims[3], dims[4])) != AFID_OK) return s;
    if (time_out) *time_out = t;
    return AFID_OK;
  });
}

// ---- mean profiles file ----------------------------------------------------------------------
extern "C" int afid_write_means(const char *dir, double tout, int nsamples, const double *times, int nxm,
                                const double *profiles, int nxmr, const double *sal_profiles) {
  return afid_guard([&]() -> int {
    static const char *const kNames[AFID_NUM_PROFILES] = {"Tbar",  "vybar", "vzbar", "vxT",  "vyT",
                                                          "vzT",   "Trms",  "vxrms", "vyrms", "vzrms",
                                                          "vxvy",  "vxvz",  "vyvz",  "chiT", "epsilon"};
    static const char *const kSalNames[AFID_NUM_SAL_PROFILES] = {"Sbar", "Srms", "vxS", "vyS", "vzS", "chiS"};
    if (!dir || nsamples < 0 || nxm < 1 || !(tout > 0.0)) return AFID_E_INVALID;
    if (nsamples > 0 && (!times || !profiles)) return AFID_E_INVALID;
    const bool sal = sal_profiles != nullptr;
    if (sal && nxmr < 1) return AFID_E_INVALID;
    if (!ensure_dir(dir)) return AFID_E_IO;
    // sample names: nint(time / TOUT) as i5.5 (CalcMeanProfiles.F90:209).  A later sample with
    // the same number replaces the earlier one: HdfSerialWriteReal1D deletes an existing dataset
    // of that name before it writes (h5tools/HdfRoutines.F90:159-161).
    std::vector<std::string> stamp(nsamples);
    std::vector<int> last(100000, -1), keep;
    for (int s = 0; s < nsamples; ++s) {
      const double fr = std::round(times[s] / tout);
      if (!(fr >= 0.0 && fr <= 99999.0)) return AFID_E_INVALID;
      last[(size_t)fr] = s;
      char b[8];
      std::snprintf(b, sizeof(b), "%05d", (int)fr);
      stamp[s] = b;
    }
    for (int s = 0; s < nsamples; ++s)
      if (last[(size_t)std::round(times[s] / tout)] == s) keep.push_back(s);
    const int ngroups = AFID_NUM_PROFILES + (sal ? AFID_NUM_SAL_PROFILES : 0);
    std::vector<std::string> names;
    names.reserve((size_t)ngroups * (keep.size() + 1));
    std::vector<afid_h5_dataset_t> sets;
    sets.reserve(names.capacity());
    auto add = [&](std::string name, int dtype, int64_t len, const double *data) {
      names.push_back(std::move(name));
      afid_h5_dataset_t d{};
      d.dtype = dtype;
      d.rank = 1;
      d.dims[0] = len;
      d.data = data;
      sets.push_back(d);
    };
    for (int q = 0; q < ngroups; ++q) {  // HdfCreateMeansFile / CreateSalinityH5Groups: the groups
      const bool sq = q >= AFID_NUM_PROFILES;
      const char *g = sq ? kSalNames[q - AFID_NUM_PROFILES] : kNames[q];
      add(g, AFID_H5_GROUP, 0, nullptr);
      for (int s : keep) {
        const double *src = sq ? sal_profiles + ((size_t)s * AFID_NUM_SAL_PROFILES + (q - AFID_NUM_PROFILES)) * nxmr
                               : profiles + ((size_t)s * AFID_NUM_PROFILES + q) * nxm;
        add(std::string(g) + "/" + stamp[s], AFID_H5_F64, sq ? nxmr : nxm, src);
      }
    }
    for (size_t i = 0; i < sets.size(); ++i) sets[i].name = names[i].c_str();
    return afid_h5_write((std::string(dir) + "/means.h5").c_str(), (int)sets.size(), sets.data());
  });
}

// ---- movie planes --------------------------------------------------------------------------
namespace {
// The frame files of write_H5_plane (h5tools/h5_tools.F90:67-136) for one plane orientation
// (axis 0: x = const, 1: y = const or y-mean, 2: z = const or z-mean), into <dir>/flowmov/<file>.
int write_plane_frames(const char *dir, const char *file, int axis, double tframe, int nframes, const double *times,
                       int nxm, int nym, int nzm, const double *planes, int nxmr, int nymr, int nzmr,
                       const double *sal_planes) {
  return afid_guard([&]() -> int {
    static const char *const kVars[4] = {"vx", "vy", "vz", "temp"};
    if (!dir || axis < 0 || axis > 2 || nframes < 0 || !(tframe > 0.0) || nxm < 1 || nym < 1 || nzm < 1)
      return AFID_E_INVALID;
    if (nframes > 0 && (!times || !planes)) return AFID_E_INVALID;
    const bool sal = sal_planes != nullptr;
    if (sal && (nxmr < 1 || nymr < 1 || nzmr < 1)) return AFID_E_INVALID;
    const int nx = nxm + 1;
    // a plane as afid_gpu_slice returns it: (rows, cols) with cols the fastest index
    const int rows = axis == 2 ? nym : nzm, cols = axis == 0 ? nym : nx;
    const size_t plane = (size_t)rows * cols;
    const int rrows = axis == 2 ? nymr : nzmr, rcols = axis == 0 ? nymr : nxmr;
    const size_t rplane = (size_t)rrows * rcols;
    std::string d = dir;
    if (!ensure_dir(d) || !ensure_dir(d + "/flowmov")) return AFID_E_IO;
    // frame numbers nint(time / TFRAME); a later frame with the same number replaces the earlier
    // one, as the reference deletes an existing dataset before writing it (h5_tools.F90:117-118)
    std::vector<int> frame(nframes), keep;
    std::vector<int> last(100000, -1);
    for (int f = 0; f < nframes; ++f) {
      const double fr = std::round(times[f] / tframe);
      if (!(fr >= 0.0 && fr <= 99999.0)) return AFID_E_INVALID;
      frame[f] = (int)fr;
      last[(size_t)fr] = f;
    }
    for (int f = 0; f < nframes; ++f)
      if (last[(size_t)frame[f]] == f) keep.push_back(f);
    // the files hold nxm rows of the cell-centred fields in the y and z cuts (nx for vx)
    std::vector<std::vector<double>> trimmed;
    trimmed.reserve(keep.size() * 3);
    std::vector<std::string> names;
    std::vector<afid_h5_dataset_t> sets;
    const int ngroups = 4 + (sal ? 1 : 0);
    names.reserve((size_t)ngroups * (keep.size() + 1));
    sets.reserve(names.capacity());
    auto add = [&](std::string name, int dtype, int64_t d0, int64_t d1, const double *data) {
      names.push_back(std::move(name));
      afid_h5_dataset_t e{};
      e.dtype = dtype;
      e.rank = 2;
      e.dims[0] = d0;
      e.dims[1] = d1;
      e.data = data;
      sets.push_back(e);
    };
    for (int v = 0; v < ngroups; ++v) {  // h5_add_slice_groups
      const char *g = v < 4 ? kVars[v] : "sal";
      add(g, AFID_H5_GROUP, 0, 0, nullptr);
      for (int f : keep) {
        char b[8];
        std::snprintf(b, sizeof(b), "%05d", frame[f]);
        const std::string name = std::string(g) + "/" + b;
        if (v == 4) {
          add(name, AFID_H5_F64, rrows, rcols, sal_planes + (size_t)f * rplane);
        } else if (axis == 0 || v == 0) {
          add(name, AFID_H5_F64, rows, cols, planes + ((size_t)f * 4 + v) * plane);
        } else {  // vy, vz, temp of the y and z cuts: rows of nxm
          const double *src = planes + ((size_t)f * 4 + v) * plane;
          trimmed.emplace_back((size_t)rows * nxm);
          for (int r = 0; r < rows; ++r)
            std::memcpy(&trimmed.back()[(size_t)r * nxm], src + (size_t)r * cols, sizeof(double) * nxm);
          add(name, AFID_H5_F64, rows, nxm, trimmed.back().data());
        }
      }
    }
    for (size_t i = 0; i < sets.size(); ++i) sets[i].name = names[i].c_str();
    return afid_h5_write((d + "/flowmov/" + file).c_str(), (int)sets.size(), sets.data());
  });
}
}  // namespace

extern "C" int afid_write_movie(const char *dir, int axis, double tframe, int nframes, const double *times,
                                int nxm, int nym, int nzm, const double *planes, int nxmr, int nymr, int nzmr,
                                const double *sal_planes) {
  static const char *const kFile[3] = {"movie_xcut.h5", "movie_ycut.h5", "movie_zcut.h5"};
  if (axis < 0 || axis > 2) return AFID_E_INVALID;
  return write_plane_frames(dir, kFile[axis], axis, tframe, nframes, times, nxm, nym, nzm, planes, nxmr, nymr,
                            nzmr, sal_planes);
}

// mean_yplane / mean_zplane (h5tools/mean_zplane.F90:131-258 / 2-129): the same layout as the
// y and z cuts, in flowmov/movie_ymean.h5 and flowmov/movie_zmean.h5.
extern "C" int afid_write_movie_mean(const char *dir, int axis, double tframe, int nframes, const double *times,
                                     int nxm, int nym, int nzm, const double *planes, int nxmr, int nymr, int nzmr,
                                     const double *sal_planes) {
  if (axis != 1 && axis != 2) return AFID_E_INVALID;
  return write_plane_frames(dir, axis == 1 ? "movie_ymean.h5" : "movie_zmean.h5", axis, tframe, nframes, times, nxm,
                            nym, nzm, planes, nxmr, nymr, nzmr, sal_planes);
}

// write_3D_spectrum (h5tools/h5_tools.F90:229-302): dataset 'var' declared (nxm, nym, nzm) in
// Fortran order; the nym/2 + 1 computed wavenumber rows fill its first rows (the hyperslab of
// the spectral decomposition) and the rest keep the fill value 0.
extern "C" int afid_write_spectrum(const char *path, int nxm, int nym, int nzm, const double *half) {
  return afid_guard([&]() -> int {
    if (!path || !half || nxm < 1 || nym < 2 || nzm < 1) return AFID_E_INVALID;
    const int nyh = nym / 2 + 1;
    std::vector<double> full((size_t)nzm * nym * nxm, 0.0);
    for (int i = 0; i < nzm; ++i)
      std::memcpy(&full[(size_t)i * nym * nxm], half + (size_t)i * nyh * nxm, sizeof(double) * (size_t)nyh * nxm);
    afid_h5_dataset_t d{};
    d.name = "var";
    d.dtype = AFID_H5_F64;
    d.rank = 3;
    d.dims[0] = nzm;
    d.dims[1] = nym;
    d.dims[2] = nxm;
    d.data = full.data();
    return afid_h5_write(path, 1, &d);
  });
}

// ---- grid coordinates ----------------------------------------------------------------------
extern "C" int afid_write_grid_info(const char *dir, const afid_tables_t *t, const afid_mgrd_t *m) {
  return afid_guard([&]() -> int {
    if (!dir || !t) return AFID_E_INVALID;
    const afid_grid_t *g = afid_tables_grid(t);
    if (!g) return AFID_E_INVALID;
    const int nxm = g->nxm, nym = g->nym, nzm = g->nzm;
    struct Item {
      const char *name;
      const char *table;
      int count;
      bool refined;
    };
    std::vector<Item> items = {{"xm", "xm", nxm, false}, {"xc", "xc", nxm + 1, false},
                               {"ym", "ym", nym, false}, {"zm", "zm", nzm, false}};
    if (m) {
      const afid_sal_grid_t *v = afid_mgrd_view(m);
      items.push_back({"xmr", "xmr", v->nxmr, true});
      items.push_back({"xcr", "xcr", v->nxmr + 1, true});
      items.push_back({"ymr", "ymr", v->nymr, true});
      items.push_back({"zmr", "zmr", v->nzmr, true});
    }
    std::vector<afid_h5_dataset_t> sets;
    for (const Item &it : items) {
      int len = 0;
      const double *a = it.refined ? afid_mgrd_array(m, it.table, &len) : afid_tables_array(t, it.table, &len);
      if (!a || len < it.count) return AFID_E_INVALID;
      afid_h5_dataset_t d{};
      d.name = it.name;
      d.dtype = AFID_H5_F64;
      d.rank = 1;
      d.dims[0] = it.count;
      d.data = a;
      sets.push_back(d);
    }
    if (!ensure_dir(dir)) return AFID_E_IO;
    return afid_h5_write((std::string(dir) + "/cordin_info.h5").c_str(), (int)sets.size(), sets.data());
  });
}
