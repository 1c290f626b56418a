// libhos_hostshim.so: single-rank MPI, the FFTW-MPI set-up calls and the
// HDF5 calls of the reference's host driver (Csource/2dpar/main_2d_par.c,
// hdf5_routines_2d_par.c, xdmf_routines_2d_par.c), so that the driver builds
// unchanged and runs against libhos_gpu.so on a host that has none of MPI,
// FFTW or libhdf5.  The headers in include/ declare what is offered and its
// limits; the HDF5 calls sit on the library's own format subset (hos_h5_*).
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "fftw3-mpi.h"
#include "hdf5.h"
#include "hos_gpu.h"

// ---------------------------------------------------------------- MPI
extern "C" {

int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Init_thread(int*, char***, int required, int* provided) {
  if (provided) *provided = required;
  return MPI_SUCCESS;
}
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int* size) {
  *size = 1;
  return MPI_SUCCESS;
}
int MPI_Comm_rank(MPI_Comm, int* rank) {
  *rank = 0;
  return MPI_SUCCESS;
}
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op, int, MPI_Comm) {
  const size_t es = type == MPI_FLOAT ? sizeof(float) : type == MPI_INT ? sizeof(int) : sizeof(double);
  if (sendbuf != recvbuf) std::memmove(recvbuf, sendbuf, es * (size_t)count);
  return MPI_SUCCESS;
}

}  // extern "C"

// ---------------------------------------------------------------- FFTW-MPI set-up
struct hos_hostshim_plan {
  ptrdiff_t n0, n1;
  int kind;  // 0 r2c, 1 c2r
};

namespace {
void* aligned(size_t bytes) {
  void* p = nullptr;
  if (posix_memalign(&p, 64, bytes ? bytes : 64) != 0) return nullptr;
  return p;
}
}  // namespace

extern "C" {

void fftw_mpi_init(void) {}
void fftw_mpi_cleanup(void) {}
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int) {}

// One rank holds the whole grid: n0 rows of n1 complex values.
ptrdiff_t fftw_mpi_local_size_2d(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm, ptrdiff_t* local_n0,
                                 ptrdiff_t* local_0_start) {
  *local_n0 = n0;
  *local_0_start = 0;
  return n0 * n1;
}

// The transposed-out spectrum [n1][n0] of one rank (n1 = Ny/2+1 as the
// driver passes it, main_2d_par.c:143).
ptrdiff_t fftw_mpi_local_size_2d_transposed(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm, ptrdiff_t* local_n0,
                                            ptrdiff_t* local_0_start, ptrdiff_t* local_n1,
                                            ptrdiff_t* local_1_start) {
  *local_n0 = n0;
  *local_0_start = 0;
  *local_n1 = n1;
  *local_1_start = 0;
  return n0 * n1;
}

double* fftw_alloc_real(size_t n) { return static_cast<double*>(aligned(n * sizeof(double))); }
fftw_complex* fftw_alloc_complex(size_t n) { return static_cast<fftw_complex*>(aligned(n * 2 * sizeof(double))); }
void fftw_free(void* p) { free(p); }
float* fftwf_alloc_real(size_t n) { return static_cast<float*>(aligned(n * sizeof(float))); }
fftwf_complex* fftwf_alloc_complex(size_t n) { return static_cast<fftwf_complex*>(aligned(n * 2 * sizeof(float))); }
void fftwf_free(void* p) { free(p); }

fftw_plan fftw_mpi_plan_dft_r2c_2d(ptrdiff_t n0, ptrdiff_t n1, double*, fftw_complex*, MPI_Comm, unsigned) {
  return new hos_hostshim_plan{n0, n1, 0};
}
fftw_plan fftw_mpi_plan_dft_c2r_2d(ptrdiff_t n0, ptrdiff_t n1, fftw_complex*, double*, MPI_Comm, unsigned) {
  return new hos_hostshim_plan{n0, n1, 1};
}
void fftw_destroy_plan(fftw_plan p) { delete p; }

void fftw_execute(const fftw_plan p) {
  std::fprintf(stderr,
               "libhos_hostshim: fftw_execute (%s %td x %td) is not available on the host; the transforms run on "
               "the GPU through fft_2d / ifft_2d of libhos_gpu.so\n",
               p && p->kind ? "c2r" : "r2c", p ? p->n0 : (ptrdiff_t)0, p ? p->n1 : (ptrdiff_t)0);
  std::exit(EXIT_FAILURE);
}

}  // extern "C"

// ---------------------------------------------------------------- HDF5 subset
namespace {

enum ObjKind { O_FILE = 1, O_DSET, O_SPACE, O_PLIST, O_TYPE };

struct Dset {
  std::string name;
  int type = HOS_H5_F64;  // stored type (created datasets)
  int rank = 0;
  long long dims[2] = {1, 1};
  std::vector<double> data;  // created datasets: the values, in double
};

struct Obj {
  explicit Obj(ObjKind k) : kind(k) {}
  ObjKind kind;
  // file
  std::string path;
  bool created = false;
  std::vector<hid_t> dsets;  // created datasets, in creation order
  // dataset
  hid_t file = 0;
  Dset d;
  // dataspace
  int rank = 0;
  long long dims[2] = {1, 1};
  bool sel = false;  // a hyperslab is selected
  long long start[2] = {0, 0}, count[2] = {1, 1};
  // datatype / property list
  hid_t type = 0;
};

std::mutex g_mu;
std::map<hid_t, Obj> g_obj;
hid_t g_next = 0x100;

int h5err(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::fprintf(stderr, "libhos_hostshim (HDF5): ");
  std::vfprintf(stderr, fmt, ap);
  std::fprintf(stderr, "\n");
  va_end(ap);
  return -1;
}

Obj* get(hid_t id, ObjKind k) {
  auto it = g_obj.find(id);
  return (it == g_obj.end() || it->second.kind != k) ? nullptr : &it->second;
}

hid_t add(Obj o) {
  const hid_t id = g_next++;
  g_obj.emplace(id, std::move(o));
  return id;
}

int type_code(hid_t t) {
  if (t == H5T_IEEE_F64LE) return HOS_H5_F64;
  if (t == H5T_IEEE_F32LE) return HOS_H5_F32;
  if (Obj* o = get(t, O_TYPE)) return type_code(o->type);
  return -1;
}

long long nelem(int rank, const long long* dims) {
  long long n = 1;
  for (int q = 0; q < rank; q++) n *= dims[q];
  return n;
}

// The block of a dataset of dims[rank] that a file-space selection names:
// start/count per dimension (the whole dataset for H5S_ALL).
int selection(hid_t file_space, int rank, const long long* dims, long long* start, long long* count) {
  for (int q = 0; q < 2; q++) {
    start[q] = 0;
    count[q] = q < rank ? dims[q] : 1;
  }
  if (file_space == H5S_ALL) return 0;
  Obj* s = get(file_space, O_SPACE);
  if (!s) return h5err("invalid file dataspace %lld", file_space);
  if (!s->sel) return 0;
  for (int q = 0; q < rank && q < 2; q++) {
    start[q] = s->start[q];
    count[q] = s->count[q];
    if (start[q] < 0 || start[q] + count[q] > dims[q]) return h5err("hyperslab outside the dataset");
  }
  return 0;
}

}  // namespace

extern "C" {

hid_t H5Fopen(const char* name, unsigned flags, hid_t) {
  std::lock_guard<std::mutex> lk(g_mu);
  (void)flags;  // read and read-write opens read the same way; this subset adds no datasets to existing files
  FILE* f = std::fopen(name, "rb");
  if (!f) return h5err("cannot open %s", name);
  std::fclose(f);
  Obj o(O_FILE);
  o.path = name;
  return add(o);
}

hid_t H5Fcreate(const char* name, unsigned flags, hid_t, hid_t) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (flags & H5F_ACC_EXCL) {
    if (FILE* f = std::fopen(name, "rb")) {
      std::fclose(f);
      return h5err("%s exists", name);
    }
  }
  Obj o(O_FILE);
  o.path = name;
  o.created = true;
  return add(o);
}

herr_t H5Fclose(hid_t file) {
  std::lock_guard<std::mutex> lk(g_mu);
  Obj* f = get(file, O_FILE);
  if (!f) return h5err("invalid file %lld", file);
  int rc = 0;
  if (f->created) {
    std::vector<const char*> names;
    std::vector<const void*> data;
    std::vector<int> types, ranks;
    std::vector<long long> dims;
    std::vector<std::vector<float>> f32;  // single-precision datasets are stored as such
    f32.reserve(f->dsets.size());
    for (hid_t id : f->dsets) {
      Obj* d = get(id, O_DSET);
      if (!d) continue;
      names.push_back(d->d.name.c_str());
      if (d->d.type == HOS_H5_F32) {
        f32.emplace_back(d->d.data.begin(), d->d.data.end());
        data.push_back(f32.back().data());
      } else {
        data.push_back(d->d.data.data());
      }
      types.push_back(d->d.type);
      ranks.push_back(d->d.rank);
      dims.push_back(d->d.dims[0]);
      dims.push_back(d->d.dims[1]);
    }
    if (hos_h5_write(f->path.c_str(), (int)names.size(), names.data(), data.data(), types.data(), ranks.data(),
                     dims.data()) != HOS_OK)
      rc = h5err("writing %s: %s", f->path.c_str(), hos_last_error());
    for (hid_t id : f->dsets) g_obj.erase(id);
  }
  g_obj.erase(file);
  return rc;
}

hid_t H5Dopen(hid_t file, const char* name, hid_t) {
  std::lock_guard<std::mutex> lk(g_mu);
  Obj* f = get(file, O_FILE);
  if (!f) return h5err("invalid file %lld", file);
  const char* nm = name[0] == '/' ? name + 1 : name;
  Obj o(O_DSET);
  o.file = file;
  o.d.name = nm;
  if (f->created) {
    for (hid_t id : f->dsets) {
      Obj* d = get(id, O_DSET);
      if (d && d->d.name == nm) return id;
    }
    return h5err("no dataset %s in %s", nm, f->path.c_str());
  }
  long long dims[4] = {1, 1, 1, 1};
  int rank = 0, type = 0;
  if (hos_h5_info(f->path.c_str(), nm, &rank, dims, &type) != HOS_OK)
    return h5err("%s", hos_last_error());
  if (rank > 2) return h5err("dataset %s has rank %d (at most 2 here)", nm, rank);
  o.d.rank = rank;
  o.d.dims[0] = rank > 0 ? dims[0] : 1;
  o.d.dims[1] = rank > 1 ? dims[1] : 1;
  o.d.type = type;
  return add(o);
}

hid_t H5Dcreate(hid_t file, const char* name, hid_t type, hid_t space, hid_t, hid_t, hid_t) {
  std::lock_guard<std::mutex> lk(g_mu);
  Obj* f = get(file, O_FILE);
  Obj* s = get(space, O_SPACE);
  if (!f || !f->created) return h5err("H5Dcreate needs a file made by H5Fcreate");
  if (!s) return h5err("invalid dataspace %lld", space);
  const int tc = type_code(type);
  if (tc != HOS_H5_F64 && tc != HOS_H5_F32) return h5err("dataset type not in the subset");
  Obj o(O_DSET);
  o.file = file;
  o.d.name = name[0] == '/' ? name + 1 : name;
  o.d.type = tc;
  o.d.rank = s->rank;
  o.d.dims[0] = s->dims[0];
  o.d.dims[1] = s->dims[1];
  o.d.data.assign((size_t)nelem(s->rank, s->dims), 0.0);
  const hid_t id = add(o);
  get(file, O_FILE)->dsets.push_back(id);
  return id;
}

herr_t H5Dread(hid_t dset, hid_t mem_type, hid_t, hid_t file_space, hid_t, void* buf) {
  std::vector<double> all;
  std::string path, nm;
  int rank;
  long long dims[2], start[2], count[2];
  int mt;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    mt = type_code(mem_type);
    Obj* d = get(dset, O_DSET);
    if (!d) return h5err("invalid dataset %lld", dset);
    Obj* f = get(d->file, O_FILE);
    if (!f) return h5err("dataset's file is closed");
    if (mt != HOS_H5_F64 && mt != HOS_H5_F32) return h5err("memory type not in the subset");
    rank = d->d.rank;
    dims[0] = d->d.dims[0];
    dims[1] = d->d.dims[1];
    if (selection(file_space, rank, dims, start, count)) return -1;
    if (f->created) {
      all = d->d.data;
    } else {
      path = f->path;
      nm = d->d.name;
    }
  }
  if (all.empty()) {
    all.resize((size_t)nelem(rank, dims));
    if (hos_h5_read_f64(path.c_str(), nm.c_str(), all.data(), (long long)all.size()) != HOS_OK)
      return h5err("%s", hos_last_error());
  }
  const long long ncol = rank > 1 ? dims[1] : 1;
  size_t k = 0;
  for (long long r = 0; r < count[0]; r++)
    for (long long c = 0; c < count[1]; c++, k++) {
      const double v = all[(size_t)((start[0] + r) * ncol + start[1] + c)];
      if (mt == HOS_H5_F64)
        static_cast<double*>(buf)[k] = v;
      else
        static_cast<float*>(buf)[k] = (float)v;
    }
  return 0;
}

herr_t H5Dwrite(hid_t dset, hid_t mem_type, hid_t, hid_t file_space, hid_t, const void* buf) {
  std::lock_guard<std::mutex> lk(g_mu);
  Obj* d = get(dset, O_DSET);
  if (!d) return h5err("invalid dataset %lld", dset);
  if (d->d.data.empty()) return h5err("H5Dwrite needs a dataset made by H5Dcreate");
  const int mt = type_code(mem_type);
  if (mt != HOS_H5_F64 && mt != HOS_H5_F32) return h5err("memory type not in the subset");
  long long start[2], count[2];
  if (selection(file_space, d->d.rank, d->d.dims, start, count)) return -1;
  const long long ncol = d->d.rank > 1 ? d->d.dims[1] : 1;
  size_t k = 0;
  for (long long r = 0; r < count[0]; r++)
    for (long long c = 0; c < count[1]; c++, k++)
      d->d.data[(size_t)((start[0] + r) * ncol + start[1] + c)] =
          mt == HOS_H5_F64 ? static_cast<const double*>(buf)[k] : (double)static_cast<const float*>(buf)[k];
  return 0;
}

hid_t H5Dget_space(hid_t dset) {
  std::lock_guard<std::mutex> lk(g_mu);
  Obj* d = get(dset, O_DSET);
  if (!d) return h5err("invalid dataset %lld", dset);
  Obj s(O_SPACE);
  s.rank = d->d.rank;
  s.dims[0] = d->d.dims[0];
  s.dims[1] = d->d.dims[1];
  return add(s);
}

herr_t H5Dclose(hid_t dset) {
  std::lock_guard<std::mutex> lk(g_mu);
  Obj* d = get(dset, O_DSET);
  if (!d) return h5err("invalid dataset %lld", dset);
  Obj* f = get(d->file, O_FILE);
  if (!f || !f->created) g_obj.erase(dset);  // a created dataset lives until its file is written
  return 0;
}

hid_t H5Screate_simple(int rank, const hsize_t* dims, const hsize_t*) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (rank < 0 || rank > 2) return h5err("dataspace of rank %d (at most 2 here)", rank);
  Obj s(O_SPACE);
  s.rank = rank;
  for (int q = 0; q < rank; q++) s.dims[q] = (long long)dims[q];
  return add(s);
}

herr_t H5Sselect_hyperslab(hid_t space, H5S_seloper_t op, const hsize_t* start, const hsize_t* stride,
                           const hsize_t* count, const hsize_t* block) {
  std::lock_guard<std::mutex> lk(g_mu);
  Obj* s = get(space, O_SPACE);
  if (!s) return h5err("invalid dataspace %lld", space);
  if (op != H5S_SELECT_SET) return h5err("only H5S_SELECT_SET selections");
  for (int q = 0; q < s->rank; q++) {
    if ((stride && stride[q] != 1) || (block && block[q] != 1)) return h5err("strided hyperslabs are not supported");
    s->start[q] = (long long)start[q];
    s->count[q] = (long long)count[q];
  }
  s->sel = true;
  return 0;
}

herr_t H5Sclose(hid_t space) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!get(space, O_SPACE)) return h5err("invalid dataspace %lld", space);
  g_obj.erase(space);
  return 0;
}

hid_t H5Pcreate(hid_t cls) {
  std::lock_guard<std::mutex> lk(g_mu);
  Obj p(O_PLIST);
  p.type = cls;
  return add(p);
}
herr_t H5Pset_fapl_mpio(hid_t, MPI_Comm, MPI_Info) { return 0; }
herr_t H5Pclose(hid_t plist) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_obj.erase(plist);
  return 0;
}

hid_t H5Tcopy(hid_t type) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (type_code(type) < 0) return h5err("datatype not in the subset");
  Obj t(O_TYPE);
  t.type = type;
  return add(t);
}
herr_t H5Tclose(hid_t type) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_obj.erase(type);
  return 0;
}

}  // extern "C"
