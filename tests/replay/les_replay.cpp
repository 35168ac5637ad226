// les_replay.cpp -- a C++ host that drives libles_gpu.so through its C ABI
// in the order the reference's program les.F90 calls the routines the
// library replaces: the caller a Fortran host becomes once the shim
// (paes-channelflow_b200/fortran/les_gpu_shim.f90) is linked in.
//
//   les.F90:146-149  setcombuf, allocate_arrays, initwave, fft_init
//                    -> les_gpu_default_config + les_gpu_init
//   les.F90:173-190  initvel + deal of every level
//                    -> les_gpu_make_ic (seeded initial field, dealt, projected)
//   les.F90:205-208  dt from the advective CFL (fixed for the run)
//                    -> les_gpu_cfl_dt
//   les.F90:203-354  time loop: xkmax (:216), mnout (:238-245), then per stage
//                    (:254-285) lower, upper, comp1, comprhs, press, comp2
//                    -> les_gpu_lower/upper/comp1/comprhs/press/comp2
//   les.F90:287-323  compmn + profile output at mnout steps -> les_gpu_stats
//   les.F90:331-351  restart file at fdout steps -> les_gpu_write_field
//   les.F90:356-357  fft_finalize, deallocate_arrays -> les_gpu_sync + les_gpu_finalize
//
// usage: les_replay nnx nny nnz re_tau nsteps meanfrq savfrq prefix
// Writes <prefix><it>.field every savfrq steps and at the end, and prints
// one line per mnout step: it, utau, utau_s, max divz, mean u at mid-height.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "les_gpu.h"

static int check(les_handle* h, int rc, const char* what) {
  if (rc != LES_OK) {
    std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, les_gpu_last_error(h));
    std::exit(2);
  }
  return rc;
}

int main(int argc, char** argv) {
  if (argc != 9) {
    std::fprintf(stderr, "usage: %s nnx nny nnz re_tau nsteps meanfrq savfrq prefix\n", argv[0]);
    return 1;
  }
  const int nnx = std::atoi(argv[1]), nny = std::atoi(argv[2]), nnz = std::atoi(argv[3]);
  const double re_tau = std::atof(argv[4]);
  const int nsteps = std::atoi(argv[5]), meanfrq = std::atoi(argv[6]), savfrq = std::atoi(argv[7]);
  const std::string prefix = argv[8];

  // RK3 coefficients (les.F90:26-27)
  const double zetas[3] = {0.0, 17.0 / 60.0, 5.0 / 12.0};
  const double gama[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};

  // namelist + derived constants (les.F90:65-121) for the channel: Lx = 2 pi,
  // Ly = pi, walls at z = 0, 2, Re_tau through the roughness z0
  les_config c;
  les_gpu_default_config(&c);
  c.nnx = nnx; c.nny = nny; c.nnz = nnz;
  c.imodel = LES_SGS_DEARDORFF; c.isurface = 6; c.precision = LES_PREC_FP64;
  c.xl = 2.0 * M_PI; c.yl = M_PI; c.zl = 2.0;
  c.z0 = std::exp(-0.4 * 5.0) * 1.0 / re_tau;
  const double utau = std::sqrt(0.016);
  const double ub = utau * ((std::log(re_tau) - 1.0) / 0.4 + 5.0);
  // the namelist's fixed dt: CFL 0.5 of the initial field (les.F90:205-208),
  // from a first handle holding that field
  double dt = 0.0;
  {
    c.dt = 1e-3;
    les_handle* t = nullptr;
    check(nullptr, les_gpu_init(&c, &t), "les_gpu_init");
    check(t, les_gpu_make_ic(t, 12345ull, ub, 0.1, utau, 1e-4), "les_gpu_make_ic");
    check(t, les_gpu_cfl_dt(t, 0.5, &dt), "les_gpu_cfl_dt");
    les_gpu_finalize(t);
  }
  c.dt = dt;
  les_handle* h = nullptr;
  check(nullptr, les_gpu_init(&c, &h), "les_gpu_init");
  // initial field (replaces initvel + deal)
  check(h, les_gpu_make_ic(h, 12345ull, ub, 0.1, utau, 1e-4), "les_gpu_make_ic");
  const double dz = c.zl / nnz;

  std::vector<double> meanbuf((size_t)19 * nnz), sc(5);
  double time = 0.0;
  for (int it = 0; it < nsteps; it++) {
    const double xkmax = dz * dz / dt / 5.0;  // les.F90:216
    time += dt;
    const bool mnout = (it == 0) || (meanfrq > 0 && it % meanfrq == 0);
    const bool fdout = (savfrq > 0 && (it + 1) % savfrq == 0) || it + 1 == nsteps;
    for (int istage = 1; istage <= 3; istage++) {
      const double dtab1 = dt * gama[istage - 1], dtab2 = dt * zetas[istage - 1], dtabm = 1.0 / dtab1;
      check(h, les_gpu_lower(h), "lower");
      check(h, les_gpu_upper(h), "upper");
      check(h, les_gpu_comp1(h, it, mnout ? 1 : 0, istage, dtab1, dtab2, xkmax), "comp1");
      check(h, les_gpu_comprhs(h, dtabm), "comprhs");
      check(h, les_gpu_press(h), "press");
      check(h, les_gpu_comp2(h, dtab1), "comp2");
    }
    if (mnout) {
      check(h, les_gpu_stats(h, meanbuf.data(), sc.data()), "compmn");
      double dmax = 0.0;
      for (int iz = 0; iz < nnz; iz++) dmax = std::fmax(dmax, meanbuf[(size_t)19 * iz + 2]);
      std::printf("%d %.17g %.17g %.17g %.17g\n", it, sc[0], sc[1], dmax, meanbuf[(size_t)19 * (nnz / 2) + 3]);
    }
    if (fdout) {
      const std::string f = prefix + std::to_string(it + 1) + ".field";
      check(h, les_gpu_write_field(h, f.c_str(), time, 8, 0), "write_field");
    }
  }
  check(h, les_gpu_sync(h, 60.0), "les_gpu_sync");
  les_gpu_finalize(h);
  std::printf("dt %.17g\n", dt);
  return 0;
}
