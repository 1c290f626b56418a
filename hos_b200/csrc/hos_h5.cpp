// HDF5 file-format subset: the files the HOS driver reads and writes,
// without libhdf5.
//
// The reference reads its parameters and initial condition with libhdf5
// (hdf5_routines_2d_par.c:13-101 get_params, :104-188 get_ic_2d) from files
// written by h5py (python/write_hdf5.py:5-40), and writes each snapshot as a
// new file of 1x1 header datasets and [Nx][Ny] fields
// (hdf5_routines_2d_par.c:227-283 write_header_2d, :286-392 write_field_2d,
// :449-537 write_extra_2d, :395-446 write_coordinates_2d).  Those files use
// the oldest layout of the format, which this file implements from the
// published HDF5 File Format Specification (version 0/1 superblock, version 1
// object headers, symbol-table groups indexed by a version 1 B-tree and a
// local heap, contiguous or compact raw data):
//
//  * reading: any dataset of the root group whose type is an IEEE float or a
//    two's-complement integer of 1-8 bytes in either byte order, converted to
//    double as H5Dread with a H5T_IEEE_F64LE memory type does; chunked or
//    filtered storage, version 2 object headers and version 2/3 superblocks
//    are reported as unsupported;
//  * writing: a new file holding datasets of the root group, each F64LE, F32LE
//    or I64LE, contiguous, with the structure libhdf5 gives such a file
//    (superblock v0, group leaf K 4 / internal K 16, one B-tree leaf over
//    symbol-table nodes of 8 entries, 256-byte object headers).
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "hos_gpu.h"

namespace hos {
void set_last_error(const char* msg);
}

namespace {

constexpr uint64_t UNDEF = ~0ull;

int h5fail(const char* path, const char* fmt, ...) {
  char msg[400], full[700];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof msg, fmt, ap);
  va_end(ap);
  snprintf(full, sizeof full, "%s: %s", path, msg);
  hos::set_last_error(full);
  return HOS_ERR_ARG;
}

int null_arg() {
  hos::set_last_error("null argument");
  return HOS_ERR_ARG;
}

// ---------------------------------------------------------------- reading
struct Dataset {
  std::string name;
  int rank = 0;
  uint64_t dims[8] = {0};
  int cls = -1;  // 0 integer, 1 float
  int size = 0;  // bytes per element
  bool big_endian = false;
  bool is_signed = true;
  int layout = -1;  // 0 compact, 1 contiguous
  uint64_t addr = UNDEF;
  uint64_t bytes = 0;
  const uint8_t* compact = nullptr;
  std::string unsupported;  // why the dataset cannot be read, if it cannot
  // element count, or UNDEF if it overflows
  uint64_t count() const {
    uint64_t n = 1;
    for (int i = 0; i < rank; i++) {
      if (dims[i] && n > UINT64_MAX / dims[i]) return UNDEF;
      n *= dims[i];
    }
    return n;
  }
};

struct File {
  const char* path = "";
  const uint8_t* p = nullptr;
  size_t len = 0;
  int fd = -1;
  uint64_t base = 0;
  int so = 8, sl = 8;  // sizes of offsets and lengths
  std::vector<Dataset> sets;
  std::string err;

  ~File() {
    if (p) munmap((void*)p, len);
    if (fd >= 0) close(fd);
  }
  bool in(uint64_t a, uint64_t n) const { return a <= len && n <= len - a; }
  uint64_t uint(uint64_t a, int n) const {
    uint64_t v = 0;
    for (int i = n - 1; i >= 0; i--) v = (v << 8) | p[a + i];
    return v;
  }
  uint64_t off(uint64_t a) const {
    uint64_t v = uint(a, so);
    if (so < 8 && v == (1ull << (8 * so)) - 1) return UNDEF;
    return v;
  }
  bool bad(const char* what) {
    if (err.empty()) err = what;
    return false;
  }
};

bool read_header(File& f, uint64_t addr, Dataset& d, uint64_t* stab_btree, uint64_t* stab_heap);

bool parse_superblock(File& f, uint64_t* root_oh, uint64_t* btree, uint64_t* heap) {
  static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  uint64_t at = UNDEF;
  for (uint64_t a = 0; a + 8 <= f.len; a = a ? a * 2 : 512) {
    if (!memcmp(f.p + a, sig, 8)) {
      at = a;
      break;
    }
  }
  if (at == UNDEF) return f.bad("no HDF5 signature");
  if (!f.in(at, 24)) return f.bad("truncated superblock");
  const int ver = f.p[at + 8];
  if (ver > 1) return f.bad("superblock version 2/3 (files written with libver='latest') are not supported");
  f.so = f.p[at + 13];
  f.sl = f.p[at + 14];
  if (f.so < 2 || f.so > 8 || f.sl < 2 || f.sl > 8) return f.bad("bad offset/length sizes");
  uint64_t a = at + 24 + (ver == 1 ? 4 : 0);
  if (!f.in(a, 4 * f.so + 2 * f.so + 8 + 16)) return f.bad("truncated superblock");
  f.base = f.off(a);
  a += 4 * f.so;  // base, free-space, end-of-file, driver addresses
  // root group symbol table entry: name offset, object header, cache type, reserved, scratch
  a += f.so;
  *root_oh = f.off(a) + f.base;
  const uint32_t cache = (uint32_t)f.uint(a + f.so, 4);
  *btree = *heap = UNDEF;
  if (cache == 1) {
    *btree = f.off(a + f.so + 8) + f.base;
    *heap = f.off(a + f.so + 8 + f.so) + f.base;
  }
  return true;
}

// Names and object headers of the root group's members, walking the v1
// B-tree of a symbol-table group down to its symbol-table nodes.
bool walk_btree(File& f, uint64_t node, uint64_t heap_data, uint64_t heap_len, int depth,
                std::vector<std::pair<std::string, uint64_t>>& out) {
  if (depth > 16) return f.bad("B-tree too deep");
  if (!f.in(node, 8 + 2 * f.so)) return f.bad("B-tree node out of the file");
  if (memcmp(f.p + node, "TREE", 4)) return f.bad("bad B-tree signature");
  if (f.p[node + 4] != 0) return f.bad("not a group B-tree");
  const int level = f.p[node + 5];
  const int used = (int)f.uint(node + 6, 2);
  uint64_t a = node + 8 + 2 * f.so;
  for (int i = 0; i < used; i++) {
    const uint64_t child_at = a + f.sl + (uint64_t)i * (f.sl + f.so);
    if (!f.in(child_at, f.so)) return f.bad("B-tree node truncated");
    const uint64_t child = f.off(child_at) + f.base;
    if (level > 0) {
      if (!walk_btree(f, child, heap_data, heap_len, depth + 1, out)) return false;
      continue;
    }
    if (!f.in(child, 8) || memcmp(f.p + child, "SNOD", 4)) return f.bad("bad symbol-table node");
    const int nsym = (int)f.uint(child + 6, 2);
    const uint64_t esz = 2 * f.so + 24;
    for (int k = 0; k < nsym; k++) {
      const uint64_t e = child + 8 + k * esz;
      if (!f.in(e, esz)) return f.bad("symbol-table node truncated");
      const uint64_t name_off = f.uint(e, f.so);
      const uint64_t oh = f.off(e + f.so) + f.base;
      if (name_off >= heap_len) return f.bad("name outside the local heap");
      const char* s = (const char*)f.p + heap_data + name_off;
      const size_t n = strnlen(s, heap_len - name_off);
      out.emplace_back(std::string(s, n), oh);
    }
  }
  return true;
}

bool parse_messages(File& f, uint64_t start, uint64_t end, Dataset& d, uint64_t* bt, uint64_t* hp,
                    std::vector<std::pair<uint64_t, uint64_t>>& more) {
  uint64_t a = start;
  while (a + 8 <= end) {
    const int type = (int)f.uint(a, 2);
    const uint64_t sz = f.uint(a + 2, 2);
    const uint64_t m = a + 8;
    if (m + sz > end || !f.in(m, sz)) return f.bad("object header message out of bounds");
    // every field read below lies inside the message's sz bytes
    auto need = [&](uint64_t n) { return n <= sz; };
    switch (type) {
      case 0x0001: {  // dataspace
        if (!need(4)) return f.bad("dataspace message too short");
        const int ver = f.p[m];
        d.rank = f.p[m + 1];
        if (d.rank > 8) return f.bad("dataspace rank above 8");
        const uint64_t dims_at = m + (ver == 1 ? 8 : 4);
        if (!need((ver == 1 ? 8 : 4) + (uint64_t)d.rank * f.sl)) return f.bad("dataspace truncated");
        if (ver == 2 && f.p[m + 3] == 2) d.rank = 0;  // null dataspace
        for (int i = 0; i < d.rank; i++) d.dims[i] = f.uint(dims_at + (uint64_t)i * f.sl, f.sl);
        break;
      }
      case 0x0003: {  // datatype
        if (!need(8)) return f.bad("datatype message too short");
        const int cls = f.p[m] & 0x0f;
        const int bits0 = f.p[m + 1];
        d.size = (int)f.uint(m + 4, 4);
        d.big_endian = bits0 & 1;
        if (cls == 0) {
          d.cls = 0;
          d.is_signed = bits0 & 0x08;
          if (d.size < 1 || d.size > 8) d.unsupported = "integer size";
        } else if (cls == 1) {
          d.cls = 1;
          if (d.size != 4 && d.size != 8) d.unsupported = "float size";
          if (bits0 & 0x40) d.unsupported = "VAX float order";
        } else {
          d.unsupported = "datatype class " + std::to_string(cls);
        }
        break;
      }
      case 0x0008: {  // data layout
        if (!need(2)) return f.bad("layout message too short");
        const int ver = f.p[m];
        if (ver == 3 || ver == 4) {
          d.layout = f.p[m + 1];
          if (d.layout == 0) {
            if (!need(4)) return f.bad("layout message too short");
            d.bytes = f.uint(m + 2, 2);
            if (!need(4 + d.bytes)) return f.bad("compact data outside its message");
            d.compact = f.p + m + 4;
          } else if (d.layout == 1) {
            if (!need(2 + (uint64_t)f.so + f.sl)) return f.bad("layout message too short");
            d.addr = f.off(m + 2);
            d.bytes = f.uint(m + 2 + f.so, f.sl);
          } else {
            d.unsupported = "chunked or virtual storage";
          }
        } else if (ver == 1 || ver == 2) {
          if (!need(8)) return f.bad("layout message too short");
          const int nd = f.p[m + 1];
          d.layout = f.p[m + 2];
          uint64_t q = 8;
          if (d.layout != 0) {
            if (!need(q + f.so)) return f.bad("layout message too short");
            d.addr = f.off(m + q);
            q += f.so;
          }
          q += 4ull * nd;
          if (d.layout == 0) {
            if (!need(q + 4)) return f.bad("layout message too short");
            d.bytes = f.uint(m + q, 4);
            if (!need(q + 4 + d.bytes)) return f.bad("compact data outside its message");
            d.compact = f.p + m + q + 4;
          } else if (d.layout != 1) {
            d.unsupported = "chunked storage";
          }
        } else {
          d.unsupported = "layout message version";
        }
        break;
      }
      case 0x000b:
        d.unsupported = "filtered storage";
        break;
      case 0x0010:  // continuation
        if (!need((uint64_t)f.so + f.sl)) return f.bad("continuation message too short");
        more.emplace_back(f.off(m) + f.base, f.uint(m + f.so, f.sl));
        break;
      case 0x0011:  // symbol table (a group)
        if (!need(2ull * f.so)) return f.bad("symbol table message too short");
        *bt = f.off(m) + f.base;
        *hp = f.off(m + f.so) + f.base;
        break;
      default:
        break;
    }
    a = m + sz;
  }
  return true;
}

bool read_header(File& f, uint64_t addr, Dataset& d, uint64_t* bt, uint64_t* hp) {
  if (!f.in(addr, 16)) return f.bad("object header out of the file");
  if (!memcmp(f.p + addr, "OHDR", 4)) return f.bad("version 2 object headers are not supported");
  if (f.p[addr] != 1) return f.bad("unknown object header version");
  const uint64_t hsz = f.uint(addr + 8, 4);
  std::vector<std::pair<uint64_t, uint64_t>> blocks{{addr + 16, hsz}};
  for (size_t i = 0; i < blocks.size() && i < 64; i++) {
    if (!f.in(blocks[i].first, blocks[i].second)) return f.bad("object header block out of the file");
    if (!parse_messages(f, blocks[i].first, blocks[i].first + blocks[i].second, d, bt, hp, blocks)) return false;
  }
  return true;
}

bool open_file(File& f, const char* path) {
  f.path = path;
  f.fd = open(path, O_RDONLY);
  if (f.fd < 0) return f.bad("cannot open");
  struct stat st;
  if (fstat(f.fd, &st) || st.st_size < 64) return f.bad("not an HDF5 file (too short)");
  f.len = (size_t)st.st_size;
  void* m = mmap(nullptr, f.len, PROT_READ, MAP_PRIVATE, f.fd, 0);
  if (m == MAP_FAILED) return f.bad("mmap failed");
  f.p = (const uint8_t*)m;
  uint64_t root = 0, bt = UNDEF, hp = UNDEF;
  if (!parse_superblock(f, &root, &bt, &hp)) return false;
  Dataset rootd;
  if (!read_header(f, root, rootd, &bt, &hp)) return false;
  if (bt == UNDEF || hp == UNDEF) return f.bad("root group has no symbol table");
  if (!f.in(hp, 8 + 2 * f.sl + f.so) || memcmp(f.p + hp, "HEAP", 4)) return f.bad("bad local heap");
  const uint64_t heap_len = f.uint(hp + 8, f.sl);
  const uint64_t heap_data = f.off(hp + 8 + 2 * f.sl) + f.base;
  if (!f.in(heap_data, heap_len)) return f.bad("local heap data out of the file");
  std::vector<std::pair<std::string, uint64_t>> members;
  if (!walk_btree(f, bt, heap_data, heap_len, 0, members)) return false;
  for (auto& m : members) {
    Dataset d;
    d.name = m.first;
    uint64_t b2 = UNDEF, h2 = UNDEF;
    if (!read_header(f, m.second, d, &b2, &h2)) return false;
    if (b2 != UNDEF) continue;  // a subgroup
    f.sets.push_back(d);
  }
  return true;
}

const Dataset* find(const File& f, const char* name) {
  if (name[0] == '/') name++;
  for (const Dataset& d : f.sets)
    if (d.name == name) return &d;
  return nullptr;
}

double element(const uint8_t* q, const Dataset& d) {
  uint8_t b[8];
  for (int i = 0; i < d.size; i++) b[i] = d.big_endian ? q[d.size - 1 - i] : q[i];
  if (d.cls == 1) {
    if (d.size == 8) {
      double v;
      memcpy(&v, b, 8);
      return v;
    }
    float v;
    memcpy(&v, b, 4);
    return v;
  }
  uint64_t u = 0;
  for (int i = d.size - 1; i >= 0; i--) u = (u << 8) | b[i];
  if (d.is_signed && d.size < 8 && (u >> (8 * d.size - 1)) & 1) u |= ~0ull << (8 * d.size);
  return d.is_signed ? (double)(int64_t)u : (double)u;
}

// ---------------------------------------------------------------- writing
struct Out {
  std::vector<uint8_t> b;
  void put(uint64_t at, uint64_t v, int n) {
    if (b.size() < at + n) b.resize(at + n, 0);
    for (int i = 0; i < n; i++) b[at + i] = (uint8_t)(v >> (8 * i));
  }
  void bytes(uint64_t at, const void* s, size_t n) {
    if (b.size() < at + n) b.resize(at + n, 0);
    memcpy(b.data() + at, s, n);
  }
  uint64_t grow(uint64_t n, uint64_t align = 8) {
    uint64_t at = (b.size() + align - 1) / align * align;
    b.resize(at + n, 0);
    return at;
  }
};

constexpr int LEAF_K = 4, INTERNAL_K = 16;
constexpr uint64_t SNOD_BYTES = 8 + 2 * LEAF_K * 40;
constexpr uint64_t BTREE_BYTES = 24 + (2 * INTERNAL_K + 1) * 8 + 2 * INTERNAL_K * 8;
constexpr uint64_t OH_MSG_BYTES = 256;

// One v1 message header + body at `at`; returns the next message position.
uint64_t message(Out& o, uint64_t at, int type, int flags, const std::vector<uint8_t>& body) {
  const uint64_t sz = (body.size() + 7) / 8 * 8;
  o.put(at, type, 2);
  o.put(at + 2, sz, 2);
  o.put(at + 4, flags, 1);
  o.bytes(at + 8, body.data(), body.size());
  return at + 8 + sz;
}

void le(std::vector<uint8_t>& v, uint64_t x, int n) {
  for (int i = 0; i < n; i++) v.push_back((uint8_t)(x >> (8 * i)));
}

}  // namespace

extern "C" {

int hos_h5_list(const char* path, char* names, int cap, int* count) {
  if (!path || !count) return null_arg();
  File f;
  if (!open_file(f, path)) return h5fail(path, "%s", f.err.c_str());
  std::string all;
  for (const Dataset& d : f.sets) all += d.name + "\n";
  *count = (int)f.sets.size();
  if (names && cap > 0) {
    const size_t n = std::min(all.size(), (size_t)cap - 1);
    memcpy(names, all.data(), n);
    names[n] = 0;
  }
  return HOS_OK;
}

int hos_h5_info(const char* path, const char* name, int* rank, long long* dims, int* type) {
  if (!path || !name || !rank || !dims) return null_arg();
  File f;
  if (!open_file(f, path)) return h5fail(path, "%s", f.err.c_str());
  const Dataset* d = find(f, name);
  if (!d) return h5fail(path, "no dataset '%s'", name);
  if (d->rank > 4) return h5fail(path, "dataset '%s': rank %d (at most 4 supported)", name, d->rank);
  *rank = d->rank;
  for (int i = 0; i < d->rank && i < 4; i++) dims[i] = (long long)d->dims[i];
  if (type) {
    *type = d->cls == 1 ? (d->size == 8 ? HOS_H5_F64 : HOS_H5_F32) : (d->size == 8 ? HOS_H5_I64 : HOS_H5_I32);
    if (d->cls == 0 && d->size != 8 && d->size != 4) *type = -1;
  }
  return HOS_OK;
}

int hos_h5_read_f64(const char* path, const char* name, double* out, long long nelems) {
  if (!path || !name || (!out && nelems)) return null_arg();
  File f;
  if (!open_file(f, path)) return h5fail(path, "%s", f.err.c_str());
  const Dataset* d = find(f, name);
  if (!d) return h5fail(path, "no dataset '%s'", name);
  if (!d->unsupported.empty()) return h5fail(path, "dataset '%s': %s not supported", name, d->unsupported.c_str());
  if (d->cls < 0 || d->layout < 0) return h5fail(path, "dataset '%s' has no type or layout", name);
  const uint64_t n = d->count();
  if (n == UNDEF || n > UINT64_MAX / (uint64_t)d->size) return h5fail(path, "dataset '%s': size overflows", name);
  if ((uint64_t)nelems != n) return h5fail(path, "dataset '%s' holds %llu elements, caller expects %lld", name,
                                           (unsigned long long)n, nelems);
  const uint64_t need = n * d->size;
  const uint8_t* src = nullptr;
  if (d->layout == 0) {
    if (d->bytes < need) return h5fail(path, "compact dataset '%s' is short", name);
    src = d->compact;
  } else if (d->addr == UNDEF) {  // never written: the default fill value
    std::fill(out, out + n, 0.0);
    return HOS_OK;
  } else {
    const uint64_t a = d->addr + f.base;
    if (!f.in(a, need)) return h5fail(path, "dataset '%s' extends past the end of the file", name);
    src = f.p + a;
  }
  for (uint64_t i = 0; i < n; i++) out[i] = element(src + i * d->size, *d);
  return HOS_OK;
}

int hos_h5_write(const char* path, int n, const char* const* names, const void* const* data, const int* types,
                 const int* ranks, const long long* dims) {
  if (!path || n < 0 || (n && (!names || !data || !types || !ranks || !dims)))
    return null_arg();
  const int max_sets = 2 * INTERNAL_K * 2 * LEAF_K;
  if (n > max_sets) return h5fail(path, "at most %d datasets per file", max_sets);
  std::vector<int> order(n);
  for (int i = 0; i < n; i++) {
    order[i] = i;
    if (!names[i] || !names[i][0] || strchr(names[i], '/')) return h5fail(path, "bad dataset name");
    if (ranks[i] < 0 || ranks[i] > 2) return h5fail(path, "dataset '%s': rank %d (0..2 supported)", names[i], ranks[i]);
    if (types[i] != HOS_H5_F64 && types[i] != HOS_H5_F32 && types[i] != HOS_H5_I64)
      return h5fail(path, "dataset '%s': type %d not supported for writing", names[i], types[i]);
    for (int j = 0; j < i; j++)
      if (!strcmp(names[i], names[j])) return h5fail(path, "dataset '%s' twice", names[i]);
  }
  // members of a symbol-table group are kept in name order (strcmp)
  std::sort(order.begin(), order.end(), [&](int a, int b) { return strcmp(names[a], names[b]) < 0; });

  Out o;
  o.b.resize(96);  // superblock
  const uint64_t root_oh = o.grow(16 + 24);
  const uint64_t btree = o.grow(BTREE_BYTES);
  const uint64_t heap = o.grow(32);
  // heap data: "" at offset 0, then each name, 8-byte aligned
  std::vector<uint64_t> name_off(n);
  uint64_t hlen = 8;
  for (int k = 0; k < n; k++) {
    name_off[order[k]] = hlen;
    hlen += (strlen(names[order[k]]) + 1 + 7) / 8 * 8;
  }
  const uint64_t heap_data = o.grow(hlen);
  for (int i = 0; i < n; i++) o.bytes(heap_data + name_off[i], names[i], strlen(names[i]));
  const int nsnod = (n + 2 * LEAF_K - 1) / (2 * LEAF_K);
  std::vector<uint64_t> snod(std::max(nsnod, 1));
  for (int s = 0; s < nsnod; s++) snod[s] = o.grow(SNOD_BYTES);
  std::vector<uint64_t> oh(n), raw(n), raw_bytes(n);
  for (int i = 0; i < n; i++) oh[i] = o.grow(16 + OH_MSG_BYTES);
  for (int i = 0; i < n; i++) {
    uint64_t cnt = 1;
    for (int r = 0; r < ranks[i]; r++) {
      if (dims[2 * i + r] < 0) return h5fail(path, "dataset '%s': negative dimension", names[i]);
      cnt *= (uint64_t)dims[2 * i + r];
    }
    const int es = types[i] == HOS_H5_F32 ? 4 : 8;
    raw_bytes[i] = cnt * es;
    raw[i] = o.grow(raw_bytes[i]);
    if (raw_bytes[i] && !data[i]) return h5fail(path, "dataset '%s': null data", names[i]);
    if (raw_bytes[i]) o.bytes(raw[i], data[i], raw_bytes[i]);  // little-endian host
  }
  const uint64_t eof = o.b.size();

  // superblock v0
  static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  o.bytes(0, sig, 8);
  const uint8_t vers[8] = {0, 0, 0, 0, 0, 8, 8, 0};
  o.bytes(8, vers, 8);
  o.put(16, LEAF_K, 2);
  o.put(18, INTERNAL_K, 2);
  o.put(20, 0, 4);
  o.put(24, 0, 8);      // base address
  o.put(32, UNDEF, 8);  // free-space info
  o.put(40, eof, 8);
  o.put(48, UNDEF, 8);  // driver info
  o.put(56, 0, 8);      // root entry: link name offset
  o.put(64, root_oh, 8);
  o.put(72, 1, 4);  // cache type 1: scratch holds the symbol table addresses
  o.put(80, btree, 8);
  o.put(88, heap, 8);

  // root object header: one symbol-table message
  o.put(root_oh, 1, 1);
  o.put(root_oh + 2, 1, 2);
  o.put(root_oh + 4, 1, 4);
  o.put(root_oh + 8, 24, 4);
  {
    std::vector<uint8_t> st;
    le(st, btree, 8);
    le(st, heap, 8);
    message(o, root_oh + 16, 0x0011, 0, st);
  }

  // B-tree leaf over the symbol-table nodes; key i+1 = last name of child i
  o.bytes(btree, "TREE", 4);
  o.put(btree + 4, 0, 1);
  o.put(btree + 5, 0, 1);
  o.put(btree + 6, nsnod, 2);
  o.put(btree + 8, UNDEF, 8);
  o.put(btree + 16, UNDEF, 8);
  o.put(btree + 24, 0, 8);
  for (int s = 0; s < nsnod; s++) {
    const int last = std::min(n, (s + 1) * 2 * LEAF_K) - 1;
    o.put(btree + 32 + 16 * s, snod[s], 8);
    o.put(btree + 40 + 16 * s, name_off[order[last]], 8);
  }

  // local heap: no free block
  o.bytes(heap, "HEAP", 4);
  o.put(heap + 8, hlen, 8);
  o.put(heap + 16, 1, 8);  // free list: none
  o.put(heap + 24, heap_data, 8);

  for (int s = 0; s < nsnod; s++) {
    o.bytes(snod[s], "SNOD", 4);
    o.put(snod[s] + 4, 1, 1);
    const int first = s * 2 * LEAF_K, cnt = std::min(n - first, 2 * LEAF_K);
    o.put(snod[s] + 6, cnt, 2);
    for (int k = 0; k < cnt; k++) {
      const int i = order[first + k];
      const uint64_t e = snod[s] + 8 + 40 * k;
      o.put(e, name_off[i], 8);
      o.put(e + 8, oh[i], 8);
    }
  }

  for (int i = 0; i < n; i++) {
    const uint64_t a = oh[i];
    std::vector<uint8_t> space, dtype, fill, layout;
    // dataspace v1 with maximum dimensions equal to the dimensions
    le(space, 1, 1);
    le(space, ranks[i], 1);
    le(space, ranks[i] ? 1 : 0, 1);
    le(space, 0, 5);
    for (int r = 0; r < ranks[i]; r++) le(space, (uint64_t)dims[2 * i + r], 8);
    for (int r = 0; r < ranks[i]; r++) le(space, (uint64_t)dims[2 * i + r], 8);
    if (types[i] == HOS_H5_I64) {  // version 1, fixed-point, signed, little-endian
      le(dtype, 0x10, 1);
      le(dtype, 0x08, 1);
      le(dtype, 0, 2);
      le(dtype, 8, 4);
      le(dtype, 0, 2);   // bit offset
      le(dtype, 64, 2);  // precision
    } else {  // version 1, IEEE float, little-endian, implied-one mantissa
      const bool d64 = types[i] == HOS_H5_F64;
      le(dtype, 0x11, 1);
      le(dtype, 0x20, 1);
      le(dtype, d64 ? 63 : 31, 1);  // sign bit position
      le(dtype, 0, 1);
      le(dtype, d64 ? 8 : 4, 4);
      le(dtype, 0, 2);
      le(dtype, d64 ? 64 : 32, 2);
      le(dtype, d64 ? 52 : 23, 1);  // exponent location
      le(dtype, d64 ? 11 : 8, 1);   // exponent size
      le(dtype, 0, 1);              // mantissa location
      le(dtype, d64 ? 52 : 23, 1);  // mantissa size
      le(dtype, d64 ? 1023 : 127, 4);
    }
    // fill value v2: allocation late, write if set, defined with size 0 (the default)
    le(fill, 2, 1);
    le(fill, 2, 1);
    le(fill, 2, 1);
    le(fill, 1, 1);
    le(fill, 0, 4);
    // layout v3, contiguous
    le(layout, 3, 1);
    le(layout, 1, 1);
    le(layout, raw_bytes[i] ? raw[i] : UNDEF, 8);
    le(layout, raw_bytes[i], 8);
    uint64_t m = a + 16;
    m = message(o, m, 0x0001, 0, space);
    m = message(o, m, 0x0003, 1, dtype);
    m = message(o, m, 0x0005, 1, fill);
    m = message(o, m, 0x0008, 1, layout);
    const uint64_t rest = a + 16 + OH_MSG_BYTES - m;  // a null message fills the block
    o.put(m, 0, 2);
    o.put(m + 2, rest - 8, 2);
    o.put(a, 1, 1);
    o.put(a + 2, 5, 2);
    o.put(a + 4, 1, 4);
    o.put(a + 8, OH_MSG_BYTES, 4);
  }

  const std::string tmp = std::string(path) + ".part";
  FILE* fp = fopen(tmp.c_str(), "wb");
  if (!fp) return h5fail(path, "cannot create");
  const bool ok = fwrite(o.b.data(), 1, o.b.size(), fp) == o.b.size();
  if (fclose(fp) != 0 || !ok || rename(tmp.c_str(), path) != 0) {
    remove(tmp.c_str());
    return h5fail(path, "write failed");
  }
  return HOS_OK;
}

}  // extern "C"
