// hos_run: the reference's driver program (Csource/2dpar/main_2d_par.c:37-380)
// on the GPU library, with no MPI, FFTW or libhdf5.
//
// In the current directory, as the reference does, it
//   * reads initpars.h5 (get_params, hdf5_routines_2d_par.c:13-101) and
//     initdata.<runsubid>.h5 (get_ic_2d, :104-188);
//   * truncates runtime.dat and appends "%14.10f\t%.16g\n" (step-start t,
//     stage-0 Hamiltonian) for every step (time_schemes_par.c:73-93);
//   * writes data<n>.<runsubid>.h5 at t = 0 (the input fields as read) and
//     whenever floor(t(1+eps)/dtsave) advances (main_2d_par.c:271-273,
//     :307-330), and data_extra<n>.<runsubid>.h5 when saveflg > 1
//     (:284-292, :334-352: W^(M), W^(M-2) of the initial state, which the
//     reference computes once and writes unchanged every time);
//   * writes HOS_data.xmf and data_coordinates.h5 for ParaView
//     (xdmf_routines_2d_par.c:22-137);
//   * steps while t < T - eps with t advanced by repeated addition of dt
//     (time_schemes_par.c:119), eps = 1e-8 (main_2d_par.c:12-16).
// The state stays on the GPU: it comes back to the host only at a save.
//
// The reference fixes three values in its source: the HOS order (NLevs = 2,
// euler_2d_par.h:24, so M = 3), the scheme (4, midpoint RK2,
// main_2d_par.c:252) and dt (0.2, :302).  They are the defaults here; the
// optional datasets /M, /scheme and /dt of initpars.h5 replace them, and the
// options replace both:
//   hos_run [-M order] [-dt dt] [-scheme 1..5] [-fp32] [-C dir] [-q]
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "hos_gpu.h"

namespace {

constexpr double EPS = 1e-8;

bool quiet = false;

[[noreturn]] void die(const char* what) {
  fprintf(stderr, "hos_run: %s: %s\n", what, hos_last_error());
  exit(EXIT_FAILURE);
}

void ck(int rc, const char* what) {
  if (rc != HOS_OK) die(what);
}

// Whether the file holds a dataset of that name (errors reading the file
// itself surface at the first required read).
bool has(const char* file, const char* name) {
  int rank = 0, type = 0;
  long long dims[4] = {0, 0, 0, 0};
  return hos_h5_info(file, name, &rank, dims, &type) == HOS_OK;
}

double scalar(const char* file, const char* name) {
  double v = 0;
  int rank = 0, type = 0;
  long long dims[4] = {0, 0, 0, 0};
  ck(hos_h5_info(file, name, &rank, dims, &type), name);
  long long n = 1;
  for (int i = 0; i < rank; i++) n *= dims[i];
  if (n != 1) {
    fprintf(stderr, "hos_run: %s:/%s is not a scalar\n", file, name);
    exit(EXIT_FAILURE);
  }
  ck(hos_h5_read_f64(file, name, &v, 1), name);
  return v;
}

void field(const char* file, const char* name, std::vector<double>& out, int nx, int ny) {
  out.assign((size_t)nx * ny, 0.0);
  ck(hos_h5_read_f64(file, name, out.data(), (long long)nx * ny), name);
}

// write_header_2d + the fields of one output file
void write_file(const std::string& path, double t, double g, int nx, int ny, double lx, double ly,
                const char* n1, const double* a1, const char* n2, const double* a2, const char* n3, const double* a3) {
  const double tv = t, nxv = nx, nyv = ny;
  std::vector<const char*> names = {"time", "g", "Nx", "Ny", "Lx", "Ly", n1, n2};
  std::vector<const void*> data = {&tv, &g, &nxv, &nyv, &lx, &ly, a1, a2};
  if (n3) {
    names.push_back(n3);
    data.push_back(a3);
  }
  const int n = (int)names.size();
  std::vector<int> types(n, HOS_H5_F64), ranks(n, 2);
  std::vector<long long> dims;
  for (int i = 0; i < n; i++) {
    const bool big = i >= 6;
    dims.push_back(big ? nx : 1);
    dims.push_back(big ? ny : 1);
  }
  ck(hos_h5_write(path.c_str(), n, names.data(), data.data(), types.data(), ranks.data(), dims.data()), path.c_str());
  if (!quiet) printf("Datafile '%s' written at t=%f\n", path.c_str(), t);
}

void xml_grid(FILE* x, double t, int npts, const std::string& datafile) {
  fprintf(x, "<Grid Name=\"Cells\" GridType=\"Uniform\">\n");
  fprintf(x, "<Time Value=\"%f\"/>\n", t);
  fprintf(x, "<Topology TopologyType=\"Polyvertex\" NodesPerElement=\"%d\">\n", npts);
  fprintf(x, "</Topology>\n");
  fprintf(x, "<Geometry GeometryType=\"XY\">\n");
  fprintf(x, "<DataItem DataType=\"TYPE_DATA\" Dimensions=\"%d 2\" Format=\"HDF\">\n", npts);
  fprintf(x, "data_coordinates.h5:/xy");
  fprintf(x, "</DataItem>\n");
  fprintf(x, "</Geometry>\n");
  const char* attrs[3][2] = {{"Phi", "phi"}, {"Eta", "eta"}, {"Bathy", "bat"}};
  for (auto& a : attrs) {
    fprintf(x, "<Attribute AttributeType=\"Scalar\" Center=\"Node\" Name=\"%s\">\n", a[0]);
    fprintf(x, "<DataItem DataType=\"TYPE_DATA\" Dimensions=\"%d 1\" Format=\"HDF\">%s:/%s</DataItem>\n", npts,
            datafile.c_str(), a[1]);
    fprintf(x, "</Attribute>\n");
  }
  fprintf(x, "</Grid>\n");
}

struct Runtime {
  FILE* f = nullptr;
  std::vector<double> t, H;
  void flush(hos_handle h) {
    int n = 0;
    t.resize(1 << 16);
    H.resize(1 << 16);
    ck(hos_energy_history(h, t.data(), H.data(), (int)t.size(), &n), "energy history");
    for (int i = 0; i < n; i++) fprintf(f, "%14.10f\t%.16g\n", t[i], H[i]);
    fflush(f);
    ck(hos_clear_history(h), "energy history");
  }
};

}  // namespace

int main(int argc, char** argv) {
  int order = 3, scheme = 4, prec = HOS_PREC_FP64;
  double dt = 0.2;
  bool set_order = false, set_scheme = false, set_dt = false;
  for (int i = 1; i < argc; i++) {
    const std::string a = argv[i];
    auto next = [&]() -> const char* {
      if (i + 1 >= argc) {
        fprintf(stderr, "hos_run: %s needs a value\n", a.c_str());
        exit(EXIT_FAILURE);
      }
      return argv[++i];
    };
    if (a == "-M") {
      order = atoi(next());
      set_order = true;
    } else if (a == "-dt") {
      dt = atof(next());
      set_dt = true;
    } else if (a == "-scheme") {
      scheme = atoi(next());
      set_scheme = true;
    } else if (a == "-fp32") {
      prec = HOS_PREC_FP32;
    } else if (a == "-C") {
      if (chdir(next()) != 0) {
        perror("hos_run: -C");
        return EXIT_FAILURE;
      }
    } else if (a == "-q") {
      quiet = true;
    } else {
      fprintf(stderr, "usage: hos_run [-M order] [-dt dt] [-scheme 1..5] [-fp32] [-C dir] [-q]\n");
      return EXIT_FAILURE;
    }
  }

  Runtime rt;
  rt.f = fopen("runtime.dat", "w");
  if (!rt.f) {
    perror("hos_run: runtime.dat");
    return EXIT_FAILURE;
  }

  // get_params (hdf5_routines_2d_par.c:13-101): every value read as double
  const char* pars = "initpars.h5";
  const int nx = (int)scalar(pars, "Nx"), ny = (int)scalar(pars, "Ny");
  const double lx = scalar(pars, "Lx"), ly = scalar(pars, "Ly"), g = scalar(pars, "g");
  const int runsubid = (int)scalar(pars, "runsubid");
  const double T = scalar(pars, "T"), dtsave = scalar(pars, "dtsave");
  const int saveflg = (int)scalar(pars, "saveflg");
  int rampflg = (int)scalar(pars, "rampflg");
  if (rampflg != 0 && rampflg != 1) {
    printf("Illegal value assigned to rampflag, setting to default value (0).\n");
    rampflg = 0;
  }
  const double tramp = scalar(pars, "Tramp");
  if (!set_order && has(pars, "M")) order = (int)scalar(pars, "M");
  if (!set_scheme && has(pars, "scheme")) scheme = (int)scalar(pars, "scheme");
  if (!set_dt && has(pars, "dt")) dt = scalar(pars, "dt");
  if (!(dt > 0)) {
    fprintf(stderr, "hos_run: dt must be positive\n");
    return EXIT_FAILURE;
  }

  // file names: the reference formats runsubid into 2 bytes (one digit) and
  // the snapshot number into 5 (main_2d_par.c:45,93,112)
  char subid[2], nbuf[5];
  snprintf(subid, sizeof subid, "%d", runsubid);
  const std::string init = std::string("initdata.") + subid + ".h5";
  if (!quiet) printf("Reading initial data from:\t%s\n", init.c_str());
  auto savename = [&](const char* stem, int nfld) {
    snprintf(nbuf, sizeof nbuf, "%d", nfld);
    return std::string(stem) + nbuf + "." + subid + ".h5";
  };

  std::vector<double> eta, phi, bat;
  field(init.c_str(), "eta0", eta, nx, ny);
  field(init.c_str(), "phi0", phi, nx, ny);
  field(init.c_str(), "bat0", bat, nx, ny);

  hos_params p;
  hos_default_params(&p, nx, ny);
  p.lx = lx;
  p.ly = ly;
  p.g = g;
  p.order = order;
  p.precision = prec;
  p.rampflg = rampflg;
  p.tramp = tramp;
  p.scheme = scheme;
  hos_handle h = nullptr;
  ck(hos_create(&p, &h), "hos_create");
  double t = 0.0;
  // fft_2d + Dealias of the input (main_2d_par.c:258-262)
  ck(hos_set_state_physical(h, eta.data(), phi.data(), t), "initial state");

  int nfld = 0;
  write_file(savename("data", nfld), t, g, nx, ny, lx, ly, "eta", eta.data(), "phi", phi.data(), "bat", bat.data());

  // ParaView index (init_xml, xdmf_routines_2d_par.c:22-88)
  {
    std::vector<double> xy((size_t)nx * ny * 2);
    size_t q = 0;
    for (int j = 0; j < nx; j++)
      for (int k = 0; k < ny; k++) {
        xy[q++] = 2 * k * M_PI / ly;
        xy[q++] = 2 * j * M_PI / lx;
      }
    const char* nm[1] = {"xy"};
    const void* dd[1] = {xy.data()};
    const int ty[1] = {HOS_H5_F64}, rk[1] = {2};
    const long long dm[2] = {(long long)nx * ny, 2};
    ck(hos_h5_write("data_coordinates.h5", 1, nm, dd, ty, rk, dm), "data_coordinates.h5");
  }
  FILE* xml = fopen("HOS_data.xmf", "w");
  if (!xml) {
    perror("hos_run: HOS_data.xmf");
    return EXIT_FAILURE;
  }
  fprintf(xml, "<Xdmf>\n<Domain>\n<Grid Name=\"CellTime\" GridType=\"Collection\" CollectionType=\"Temporal\">\n");
  xml_grid(xml, t, nx * ny, "data0.1.h5");  // init_xml names this file whatever runsubid is (:74-84)

  // W^(M), W^(M-2) of the initial state in physical space (main_2d_par.c:264-268)
  std::vector<double> velwM, velwM2;
  if (saveflg > 1) {
    const size_t fs = (size_t)(ny / 2 + 1) * nx * 2;
    std::vector<double> u(2 * fs), w[4];
    for (auto& x : w) x.resize(fs);
    double t0 = 0;
    ck(hos_get_state_spectral(h, u.data(), &t0), "state");
    ck(hos_zvel(h, u.data(), w[0].data(), w[1].data(), w[2].data(), w[3].data()), "Zvel");
    velwM.resize((size_t)nx * ny);
    velwM2.resize((size_t)nx * ny);
    ck(hos_ifft_2d(h, w[0].data(), velwM.data()), "ifft");
    ck(hos_ifft_2d(h, w[1].data(), velwM2.data()), "ifft");
    write_file(savename("data_extra", nfld), t, g, nx, ny, lx, ly, "Array1", velwM.data(), "Array2", velwM2.data(),
               nullptr, nullptr);
  }

  // main loop (main_2d_par.c:298-357): the steps up to the next save run
  // back to back on the GPU
  constexpr long long FLUSH = 1 << 15;  // below the device energy record's capacity
  long long since_flush = 0;
  while (t < T - EPS) {
    long long k = 0;
    bool save = false;
    double tk = t;
    while (tk < T - EPS && !save && since_flush + k < FLUSH) {
      const double told = tk;
      tk = tk + dt;
      k++;
      save = std::floor(tk * (1 + EPS) / dtsave) > std::floor(told * (1 + EPS) / dtsave);
    }
    ck(hos_step(h, dt, (int)k), "hos_step");
    since_flush += k;
    t = tk;
    if (save || since_flush >= FLUSH || !(t < T - EPS)) {
      ck(hos_sync(h), "step");
      rt.flush(h);
      since_flush = 0;
    }
    if (save) {
      nfld++;
      ck(hos_get_state_physical(h, eta.data(), phi.data()), "state");
      const std::string name = savename("data", nfld);
      write_file(name, t, g, nx, ny, lx, ly, "eta", eta.data(), "phi", phi.data(), "bat", bat.data());
      xml_grid(xml, t, nx * ny, name);
      if (saveflg > 1)
        write_file(savename("data_extra", nfld), t, g, nx, ny, lx, ly, "Array1", velwM.data(), "Array2",
                   velwM2.data(), nullptr, nullptr);
    }
  }
  fprintf(xml, "</Grid>\n</Domain>\n</Xdmf>\n");
  fclose(xml);
  fclose(rt.f);
  hos_destroy(h);
  return EXIT_SUCCESS;
}
