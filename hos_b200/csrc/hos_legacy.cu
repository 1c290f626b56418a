// The reference's hot-path entry points (include/hos_legacy.h) over the
// handle API: the same names, signatures and global-variable interface as
// Csource/2dpar's hosm_2d_par.c, time_schemes_par.c, operators_par.c and
// fft_routines_2d_par.c, with every array operation done on the GPU.
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "hos_gpu.h"
#include "hos_legacy.h"

namespace hos {
void set_last_error(const char* msg);
}

// Globals of the reference driver that these entry points read
// (euler_2d_par.h:40-98, fft_routines_2d_par.h:17-38).  A driver that
// includes the reference headers defines them as well; its definitions take
// precedence when it links against this library.
extern "C" {
int Nx = 0;
int Ny = 0;
double Lx = 0.0;
double Ly = 0.0;
double Kx0 = 0.0;
double Ky0 = 0.0;
double g = 0.0;
int rampflg = 0;
double Tramp = 1.0;
ptrdiff_t alloc_local = 0;
ptrdiff_t local_N = 0;
ptrdiff_t local_Nyhpo = 0;
ptrdiff_t local_1_start = 0;
int mpi_rank = 0;
char runtime_data_buff[32] = "runtime.dat";
double Ham = 0.0;
}

namespace {

struct Legacy {
  hos_handle h = nullptr;
  hos_params p{};
  int scheme = HOS_MIDPOINT;  // main_2d_par.c:252 uses scheme 4
  int nlevs = -1;             // NLevs, euler_2d_par.h:24
  // Resident mode: the state sol_update_RK advanced stays on the device; the
  // host array `resident` is brought up to date only when a call here reads
  // it (host_stale) and is re-uploaded after a call here writes it.
  int resident_mode = -1;     // -1: not yet read from HOS_LEGACY_RESIDENT
  double* resident = nullptr;
  bool host_stale = false;
  double dev_t = 0.0;         // the device's time after the last step
};
Legacy L;
std::mutex mu;

int nlevs_now() {
  if (L.nlevs < 0) {
    const char* s = getenv("HOS_NLEVS");
    L.nlevs = s ? atoi(s) : 2;
  }
  return L.nlevs;
}

void report(const char* where) {
  fprintf(stderr, "libhos_gpu %s: %s\n", where, hos_last_error());
}

size_t field() { return (size_t)Nx * (size_t)(Ny / 2 + 1); }

bool resident_mode() {
  if (L.resident_mode < 0) {
    const char* s = getenv("HOS_LEGACY_RESIDENT");
    L.resident_mode = (s && s[0] == '1') ? 1 : 0;
  }
  return L.resident_mode == 1;
}

// Brings the host copy of the resident state up to date.
void sync_host(const char* where) {
  if (!L.host_stale || !L.h || !L.resident) return;
  if (hos_get_state_spectral(L.h, L.resident, nullptr) != HOS_OK) report(where);
  L.host_stale = false;
}

// Whether p points into the resident packed state (both fields).
bool in_state(const void* p) {
  if (!L.resident || !p) return false;
  const double* q = static_cast<const double*>(p);
  return q >= L.resident && q < L.resident + 4 * field();
}

// Before a call reads the host array p.
void reading(const void* p, const char* where) {
  if (in_state(p)) sync_host(where);
}

// Before a call writes the host array p: the host copy becomes the newer one.
void writing(const void* p, const char* where) {
  if (!in_state(p)) return;
  sync_host(where);
  L.resident = nullptr;
}

// The context for the current globals, created or re-created on change.
hos_handle ctx(const char* where) {
  hos_params p;
  hos_default_params(&p, Nx, Ny);
  p.lx = Lx > 0 ? Lx : (Kx0 > 0 ? 2 * M_PI / Kx0 : 2 * M_PI);
  p.ly = Ly > 0 ? Ly : (Ky0 > 0 ? 2 * M_PI / Ky0 : 2 * M_PI);
  p.g = g;
  p.order = nlevs_now() + 1;
  p.precision = HOS_PREC_FP64;
  p.rampflg = rampflg;
  p.tramp = Tramp;
  p.scheme = L.scheme;
  const ptrdiff_t fsz = (ptrdiff_t)Nx * (Ny / 2 + 1);
  if ((alloc_local && alloc_local != fsz) || local_1_start != 0 || (local_Nyhpo && local_Nyhpo != Ny / 2 + 1)) {
    hos::set_last_error("only a single rank holding the whole field is supported");
    report(where);
    return nullptr;
  }
  if (L.h && memcmp(&p, &L.p, sizeof(p)) == 0) return L.h;
  sync_host(where);  // the old context holds the newest state
  L.resident = nullptr;
  if (L.h) hos_destroy(L.h);
  L.h = nullptr;
  if (hos_create(&p, &L.h) != HOS_OK) {
    report(where);
    L.h = nullptr;
    return nullptr;
  }
  L.p = p;
  return L.h;
}

}  // namespace

extern "C" {

void hos_legacy_set_nlevs(int nlevs) {
  std::lock_guard<std::mutex> lk(mu);
  L.nlevs = nlevs;
}

void Setup_TimeScheme(int scheme_flg) {
  std::lock_guard<std::mutex> lk(mu);
  L.scheme = scheme_flg;
}

void rhs_hos_setup(void) {
  std::lock_guard<std::mutex> lk(mu);
  ctx("rhs_hos_setup");
}

void hos_legacy_set_resident(int on) {
  std::lock_guard<std::mutex> lk(mu);
  sync_host("hos_legacy_set_resident");
  L.resident = nullptr;
  L.resident_mode = on ? 1 : 0;
}

void hos_legacy_sync(void) {
  std::lock_guard<std::mutex> lk(mu);
  sync_host("hos_legacy_sync");
}

void rhs_hos_clean(void) {
  std::lock_guard<std::mutex> lk(mu);
  sync_host("rhs_hos_clean");
  L.resident = nullptr;
  if (L.h) hos_destroy(L.h);
  L.h = nullptr;
}

void sol_update_RK(double* u, double* t, double dt, char* dtflag) {
  (void)dtflag;
  std::lock_guard<std::mutex> lk(mu);
  hos_handle h = ctx("sol_update_RK");
  if (!h) return;
  const bool keep = resident_mode();
  // the state on the device is current when it is this array's, advanced by
  // our last step to the caller's time
  const bool on_device = keep && L.resident == u && L.dev_t == *t;
  if (!on_device) {
    sync_host("sol_update_RK");
    L.resident = nullptr;
    if (hos_set_state_spectral(h, u, *t)) {
      report("sol_update_RK");
      return;
    }
  }
  if (hos_step(h, dt, 1)) {
    // the device state may be partly advanced: forget it, so that the next
    // call uploads the caller's array again instead of syncing this one over it
    L.resident = nullptr;
    L.host_stale = false;
    report("sol_update_RK");
    return;
  }
  if (keep) {
    L.resident = u;
    L.host_stale = true;
    L.dev_t = *t + dt;  // the device advances t exactly so (time_schemes_par.c:119)
  } else if (hos_get_state_spectral(h, u, nullptr)) {
    report("sol_update_RK");
    return;
  }
  // the newest record of the energy history is this step's stage-0 Hamiltonian
  double tt = 0.0, hh = 0.0;
  int n = 0;
  if (hos_energy_history(h, &tt, &hh, 1, &n) == HOS_OK && n == 1) Ham = hh;
  // time_schemes_par.c:73-93: rank 0 appends the stage-0 Hamiltonian
  if (mpi_rank == 0) {
    FILE* fid = fopen(runtime_data_buff, "a+");
    if (fid == NULL) {
      perror("Unable to open runtime datafile");
      exit(EXIT_FAILURE);
    }
    fprintf(fid, "%14.10f\t%.16g\n", *t, Ham);
    fclose(fid);
  }
  t[0] = t[0] + dt;  // time_schemes_par.c:119
}

void rhs_hos(double* hrhs, double* hu, double t) {
  std::lock_guard<std::mutex> lk(mu);
  hos_handle h = ctx("rhs_hos");
  reading(hu, "rhs_hos");
  writing(hrhs, "rhs_hos");
  if (h && hos_rhs(h, hu, hrhs, t)) report("rhs_hos");
}

void rhs_test(double* hrhs, double* hu) {
  std::lock_guard<std::mutex> lk(mu);
  hos_handle h = ctx("rhs_test");
  if (!h) return;
  reading(hu, "rhs_test");
  writing(hrhs, "rhs_test");
  const size_t f = field();
  if (hos_spectral_op(h, HOS_OP_DX, hu, nullptr, hrhs) ||
      hos_spectral_op(h, HOS_OP_DY, hu + 2 * f, nullptr, hrhs + 2 * f))
    report("rhs_test");
}

void Zvel(double* hu, double* hZvelM, double* hZvelM2, double* hZvel2M, double* hZvel2M2, double t) {
  (void)t;
  std::lock_guard<std::mutex> lk(mu);
  hos_handle h = ctx("Zvel");
  reading(hu, "Zvel");
  for (double* o : {hZvelM, hZvelM2, hZvel2M, hZvel2M2}) writing(o, "Zvel");
  if (h && hos_zvel(h, hu, hZvelM, hZvelM2, hZvel2M, hZvel2M2)) report("Zvel");
}

void ZvelLinear(const double* hu, double* hZvelLinear) {
  std::lock_guard<std::mutex> lk(mu);
  hos_handle h = ctx("ZvelLinear");
  reading(hu, "ZvelLinear");
  writing(hZvelLinear, "ZvelLinear");
  if (h && hos_spectral_op(h, HOS_OP_DZ, hu + 2 * field(), nullptr, hZvelLinear)) report("ZvelLinear");
}

double Hamiltonian(const double* heta, const double* heta_t, const double* hphi) {
  std::lock_guard<std::mutex> lk(mu);
  hos_handle h = ctx("Hamiltonian");
  reading(heta, "Hamiltonian");
  reading(heta_t, "Hamiltonian");
  reading(hphi, "Hamiltonian");
  double H = 0.0;
  if (h && hos_hamiltonian(h, heta, heta_t, hphi, &H)) report("Hamiltonian");
  return H;
}

double RampFun(const double t) { return 1 - exp(-t * t / Tramp / Tramp); }  // hosm_2d_par.c:526-530

static void op1(int op, const double* a, const double* b, double* out, const char* where) {
  std::lock_guard<std::mutex> lk(mu);
  hos_handle h = ctx(where);
  reading(a, where);
  reading(b, where);
  writing(out, where);
  if (h && hos_spectral_op(h, op, a, b, out)) report(where);
}

void Dx(double* hu, double* hu_x) { op1(HOS_OP_DX, hu, nullptr, hu_x, "Dx"); }
void Dy(double* hu, double* hu_y) { op1(HOS_OP_DY, hu, nullptr, hu_y, "Dy"); }
void Dz(const double* hu, double* hu_z) { op1(HOS_OP_DZ, hu, nullptr, hu_z, "Dz"); }
void Mult(double* hu1, double* hu2, double* hprod) { op1(HOS_OP_MULT, hu1, hu2, hprod, "Mult"); }
void Sum(double* hu1, double* hu2, double* hsum) { op1(HOS_OP_SUM, hu1, hu2, hsum, "Sum"); }
void Dealias(double* hu) { op1(HOS_OP_DEALIAS, hu, nullptr, hu, "Dealias"); }

void fft_2d(double* u, double* hu, void* plan) {
  (void)plan;
  std::lock_guard<std::mutex> lk(mu);
  hos_handle h = ctx("fft_2d");
  writing(hu, "fft_2d");
  if (h && hos_fft_2d_ld(h, u, Ny + 2, hu)) report("fft_2d");
}

void ifft_2d(double* hu, double* u, void* plan) {
  (void)plan;
  std::lock_guard<std::mutex> lk(mu);
  hos_handle h = ctx("ifft_2d");
  reading(hu, "ifft_2d");
  if (h && hos_ifft_2d_ld(h, hu, u, Ny + 2)) report("ifft_2d");
}

}  // extern "C"
