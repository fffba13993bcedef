// vh_run: the reference's driver loop (NEWEST5/main.cpp:90-223) on the B200
// library, through the C ABI of include/vh.h only.
//
//   init -> write the first snapshot -> loop { step; tau += ts; max T;
//   progress line; snapshots every print interval and after the first step;
//   scenario break } -> free
//
// Scenarios are the reference's compile-time blocks made runtime choices:
//   gubser     2+1D Gubser test (maindef.h GUBSER block): 129x129, dx 0.1 fm,
//              tau0 1 fm/c, dtau 0.01, conformal EOS, eta/s 0.2,
//              tau_pi = 5 eta/(e+P), Navier-Stokes pi, mirrored ghosts;
//              stops after tau > 9 fm/c (main.cpp:196-199); --cold-plasma
//              runs the COLDPLASMA test instead (init.h:489-512, the shear
//              source without -pi/tau_pi, Source.h:371-410)
//   glauber    2+1D MC-Glauber event (b, seed), synthetic EOS table,
//              eta/s 0.08, tau_pi = 1.5 eta/P, tau0 0.6, dtau 0.02;
//              stops when max T < 120 MeV (main.cpp:201-204, GINIT block)
//   glauber3d  the same on a 3+1D Milne grid (default 161x161x41, d eta 0.25)
//   shocktube  the Cartesian default block of TXYZ5 (TXYZ5/maindef.h:35-63,
//              init.h:151-210): 10x10x101 cells of 0.1 fm, t0 = 0, dt 0.01,
//              e = 16 fm^-4 for z < 0 and 1 fm^-4 for z >= 0 at rest,
//              conformal EOS with 42.25 degrees of freedom, eta/s 0.01/(4 pi)
//   bjorken    the Bjorken block of NEWEST5 (maindef.h:195-235, init.h:283-340):
//              10x10 boost-invariant cells of 0.1 fm, e = 30 GeV/fm^3 at rest,
//              tau0 0.6, dtau 0.01, conformal EOS with 42.25 degrees of
//              freedom, eta = 0.2 s, tau_pi = 0.01 fm/c; after each step the
//              centre cell's T (fm^-1) times GEVFM/1000 goes to ./temp.txt
//              beside the tau the step started from (main.cpp:145-147);
//              stops after tau > 10 fm/c (main.cpp:199-210)
// Every run also stops at tau > 25.3 fm/c (main.cpp:211) or --tau-end.
// Snapshots use the reference's names and layouts (res/tau%2.3ffm.bin, one xy
// plane on boost-invariant grids, the full grid otherwise); with --ns each
// comes with NEWEST10's Navier-Stokes file res/NStau%2.3ffm.bin.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "vh.h"

namespace {

const double kHbarc = 0.19733;
const double kAqgp = M_PI * M_PI * (16 + 31.5) / 90;  // e = a T^4 (fm units)

struct Options {
  std::string scenario = "gubser";
  int nx = 0, ny = 0, nz = 0;
  int precision = VH_PREC_FP64;
  int max_steps = 0;        // 0: until the scenario's break
  double tau_end = 25.3;    // main.cpp:211
  double print_every = 1.0; // PFREQ (fm/c)
  int write_every = 1;      // FREQ: cell stride of the snapshots
  std::string out;          // snapshot directory ("" = no snapshots)
  double b = 7.0;
  unsigned long long seed = 0;
  double floor_gev = 0.2;    // GeV/fm^3, the library workloads' Glauber floor
  bool quiet = false;
  std::string restart;      // resume from this restart file
  std::string checkpoint;   // write a restart file at the end
  bool ns = false;          // also write res/NStau%2.3ffm.bin beside each snapshot
  bool cold = false;        // gubser: the cold-plasma test (COLDPLASMA)
};

void usage() {
  std::printf(
      "usage: vh_run [--scenario gubser|glauber|glauber3d|shocktube|bjorken] [--nx N --ny N --nz N]\n"
      "              [--precision fp64|mixed] [--steps N] [--tau-end T] [--print-every T]\n"
      "              [--out DIR] [--every FREQ] [--b B] [--seed S] [--floor E_GeV_fm3] [--quiet]\n"
      "              [--restart FILE] [--checkpoint FILE] [--ns] [--cold-plasma]\n");
}

bool parse(int argc, char** argv, Options& o) {
  for (int i = 1; i < argc; i++) {
    const std::string a = argv[i];
    auto next = [&](const char* what) -> const char* {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "vh_run: %s needs a value\n", what);
        std::exit(2);
      }
      return argv[++i];
    };
    if (a == "--help" || a == "-h") { usage(); std::exit(0); }
    else if (a == "--scenario") o.scenario = next("--scenario");
    else if (a == "--nx") o.nx = std::atoi(next("--nx"));
    else if (a == "--ny") o.ny = std::atoi(next("--ny"));
    else if (a == "--nz") o.nz = std::atoi(next("--nz"));
    else if (a == "--precision") {
      const std::string p = next("--precision");
      if (p == "fp64") o.precision = VH_PREC_FP64;
      else if (p == "mixed") o.precision = VH_PREC_MIXED;
      else { std::fprintf(stderr, "vh_run: precision %s\n", p.c_str()); return false; }
    } else if (a == "--steps") o.max_steps = std::atoi(next("--steps"));
    else if (a == "--tau-end") o.tau_end = std::atof(next("--tau-end"));
    else if (a == "--print-every") o.print_every = std::atof(next("--print-every"));
    else if (a == "--out") o.out = next("--out");
    else if (a == "--every") o.write_every = std::atoi(next("--every"));
    else if (a == "--b") o.b = std::atof(next("--b"));
    else if (a == "--seed") o.seed = std::strtoull(next("--seed"), nullptr, 10);
    else if (a == "--floor") o.floor_gev = std::atof(next("--floor"));
    else if (a == "--quiet") o.quiet = true;
    else if (a == "--restart") o.restart = next("--restart");
    else if (a == "--checkpoint") o.checkpoint = next("--checkpoint");
    else if (a == "--ns") o.ns = true;
    else if (a == "--cold-plasma") o.cold = true;
    else { std::fprintf(stderr, "vh_run: unknown option %s\n", a.c_str()); usage(); return false; }
  }
  if (o.scenario != "gubser" && o.scenario != "glauber" && o.scenario != "glauber3d" && o.scenario != "shocktube" &&
      o.scenario != "bjorken") {
    std::fprintf(stderr, "vh_run: unknown scenario %s\n", o.scenario.c_str());
    return false;
  }
  return true;
}

int fail(const char* what, vh_handle* h, int code) {
  std::fprintf(stderr, "vh_run: %s: status %d: %s\n", what, code, vh_last_error(h));
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  Options o;
  if (!parse(argc, argv, o)) return 2;
  const bool gubser = o.scenario == "gubser", three_d = o.scenario == "glauber3d";
  const bool shock = o.scenario == "shocktube";
  const bool bjorken = o.scenario == "bjorken";

  vh_config c;
  std::memset(&c, 0, sizeof c);
  c.coords = VH_COORD_MILNE;
  c.precision = o.precision;
  c.recon = VH_RECON_WENO5;
  c.minmod_theta = 1.1;
  c.hbarc = kHbarc;
  std::vector<double> eos_e, eos_p, eos_c, eos_t;
  if (shock) {
    c.coords = VH_COORD_CARTESIAN;
    c.nx = o.nx ? o.nx : 10; c.ny = o.ny ? o.ny : 10; c.nz = o.nz ? o.nz : 101; c.boost_invariant = 0;
    c.dx = c.dy = c.dz = 0.1; c.tau0 = 0.0; c.dtau = 0.01;
    c.eos_kind = VH_EOS_CONFORMAL; c.eos_a = 3 * 42.25 * M_PI * M_PI / 90;
    c.hbarc = 0.1973;
    c.etas0 = 0.01 / (4 * M_PI); c.etas_tc = 0.154; c.taupi_kind = VH_TAUPI_15_ETA_OVER_P;
  } else if (bjorken) {
    c.nx = o.nx ? o.nx : 10; c.ny = o.ny ? o.ny : 10; c.nz = 1; c.boost_invariant = 1;
    c.dx = c.dy = 0.1; c.dz = 1.0; c.tau0 = 0.6; c.dtau = 0.01;
    c.eos_kind = VH_EOS_CONFORMAL; c.eos_a = 3 * 42.25 * M_PI * M_PI / 90;
    c.hbarc = 0.1973;
    c.etas0 = 0.2; c.etas_tc = 0.154; c.taupi_kind = VH_TAUPI_CONST; c.taupi_const = 0.01;
  } else if (gubser) {
    c.nx = o.nx ? o.nx : 129; c.ny = o.ny ? o.ny : 129; c.nz = 1; c.boost_invariant = 1;
    c.dx = c.dy = 0.1; c.dz = 1.0; c.tau0 = 1.0; c.dtau = 0.01;
    c.eos_kind = VH_EOS_CONFORMAL; c.eos_a = kAqgp;
    c.etas0 = 0.2; c.etas_tc = 0.154; c.taupi_kind = VH_TAUPI_5_ETA_OVER_EPP; c.gubser_mirror = 1;
    c.cold_plasma = o.cold ? 1 : 0;
  } else {
    c.nx = o.nx ? o.nx : (three_d ? 161 : 128); c.ny = o.ny ? o.ny : c.nx;
    c.nz = three_d ? (o.nz ? o.nz : 41) : 1; c.boost_invariant = three_d ? 0 : 1;
    c.dx = c.dy = 0.1; c.dz = three_d ? 0.25 : 1.0; c.tau0 = 0.6; c.dtau = 0.02;
    const int n = 2000;
    eos_e.resize(n); eos_p.resize(n); eos_c.resize(n); eos_t.resize(n);
    if (int r = vh_eos_table_synthetic(n, 1e-3, 500.0, kAqgp, kHbarc, eos_e.data(), eos_p.data(), eos_c.data(),
                                       eos_t.data()))
      return fail("vh_eos_table_synthetic", nullptr, r);
    c.eos_kind = VH_EOS_TABLE; c.eos_n = n;
    c.eos_e = eos_e.data(); c.eos_p = eos_p.data(); c.eos_cs2 = eos_c.data(); c.eos_t = eos_t.data();
    c.etas0 = 0.08; c.etas_tc = 0.154; c.taupi_kind = VH_TAUPI_15_ETA_OVER_P;
  }

  vh_handle* h = nullptr;
  if (int r = vh_create(&c, &h)) return fail("vh_create", nullptr, r);
  int gx, gy, gz;
  vh_dims(h, &gx, &gy, &gz);
  const size_t n = (size_t)gx * gy * gz;
  std::vector<double> e(n), ux(n, 0.0), uy(n, 0.0), prevu(4 * n);
  int r;
  if (shock) {
    // cell centres z = -(nz/2) dz + (k - 3) dz, as the reference centres one rank
    for (int k = 0; k < gz; k++)
      for (size_t q = 0; q < (size_t)gx * gy; q++) {
        const double z = -((c.nz / 2) * c.dz) + (k - VH_NGHOST) * c.dz;
        e[(size_t)k * gx * gy + q] = z < 0 ? 16.0 : 1.0;
      }
    r = vh_init_profile(h, c.tau0, e.data(), ux.data(), uy.data(), nullptr, nullptr, VH_PI_ZERO, nullptr);
  } else if (bjorken) {
    for (size_t q = 0; q < n; q++) e[q] = 30.0 / c.hbarc;
    r = vh_init_profile(h, c.tau0, e.data(), ux.data(), uy.data(), nullptr, nullptr, VH_PI_ZERO, nullptr);
  } else if (gubser && o.cold) {
    // NEWEST5/init.h:489-512: the cold-plasma solution (B = 1.21) with its pi
    std::vector<double> pi5(5 * n);
    r = vh_profile_gubser_cold(c.nx, c.ny, c.dx, c.dy, 1.0, c.tau0, c.dtau, 1.21, c.eos_a, e.data(), ux.data(),
                               uy.data(), pi5.data(), prevu.data());
    if (!r) r = vh_init_profile(h, c.tau0, e.data(), ux.data(), uy.data(), nullptr, prevu.data(), VH_PI_GIVEN, pi5.data());
  } else if (gubser) {
    r = vh_profile_gubser(c.nx, c.ny, c.dx, c.dy, 1.0, c.tau0, c.dtau, 0.6, c.eos_a, kHbarc, e.data(), ux.data(),
                          uy.data(), prevu.data());
    if (!r) r = vh_init_profile(h, c.tau0, e.data(), ux.data(), uy.data(), nullptr, prevu.data(), VH_PI_NS, nullptr);
  } else {
    int npart = 0;
    r = vh_profile_glauber(c.nx, c.ny, c.nz, c.boost_invariant, c.dx, c.dy, c.dz, 208, 6.62, 0.546, 0.4, o.b, 6.4,
                           0.5, 40.0, 1.5, 1.3, o.floor_gev, kHbarc, o.seed, e.data(), &npart);
    if (!r && !o.quiet) std::printf("MC-Glauber b = %.3f fm, seed %llu: %d participants\n", o.b, o.seed, npart);
    if (!r) r = vh_init_profile(h, c.tau0, e.data(), ux.data(), uy.data(), nullptr, nullptr, VH_PI_ZERO, nullptr);
  }
  if (r) { const int code = fail("initial state", h, r); vh_destroy(h); return code; }
  double tau = c.tau0;
  if (!o.restart.empty() && (r = vh_load_checkpoint(h, o.restart.c_str(), &tau))) {
    const int code = fail("vh_load_checkpoint", h, r);
    vh_destroy(h);
    return code;
  }

  const int layout = c.boost_invariant ? VH_WRITE_XY : VH_WRITE_FULL;
  auto write = [&](double tau) -> int {
    if (o.out.empty()) return 0;
    char name[512];
    std::snprintf(name, sizeof name, "%s/tau%2.3ffm.bin", o.out.c_str(), tau);
    if (int w = vh_write(h, name, layout, o.write_every)) return w;
    if (!o.ns) return 0;
    // NEWEST10/init.h:660-661 writes the Navier-Stokes pi of the initial state
    std::snprintf(name, sizeof name, "%s/NStau%2.3ffm.bin", o.out.c_str(), tau);
    return vh_write(h, name, VH_WRITE_NS_XY, o.write_every);
  };
  if (!o.out.empty()) mkdir(o.out.c_str(), 0755);

  const double ts = c.dtau;
  // a resumed run keeps the step count and print cadence of the original one
  int l = 1 + (int)std::lround((tau - c.tau0) / ts);
  double tau_print = c.tau0 + std::floor((tau - c.tau0) / o.print_every + 1e-6) * o.print_every;
  if (o.restart.empty() && (r = write(tau))) { const int code = fail("vh_write", h, r); vh_destroy(h); return code; }
  const auto start = std::chrono::steady_clock::now();
  int status = 0;
  FILE* temp_txt = bjorken ? std::fopen("temp.txt", "w") : nullptr;
  if (bjorken && !temp_txt) { const int code = fail("temp.txt", h, VH_E_ARG); vh_destroy(h); return code; }
  std::vector<double> tcell(bjorken ? n : 0);
  const size_t centre = (size_t)(gy / 2) * gx + gx / 2;  // HydroGrid[XCM/2][YCM/2][0]
  while (true) {
    if ((r = vh_step(h, 1))) { status = fail("vh_step", h, r); break; }
    if (bjorken) {
      // main.cpp:146: tau before the increment, fmtoMev(FT(e)) / 1000
      if ((r = vh_get_primitive(h, nullptr, nullptr, tcell.data(), nullptr, nullptr))) {
        status = fail("vh_get_primitive", h, r);
        break;
      }
      std::fprintf(temp_txt, "%g  %g\n", tau, tcell[centre] * c.hbarc / 1000);
    }
    tau += ts;
    double tmax_gev = 0;
    if ((r = vh_max_temperature(h, &tmax_gev))) { status = fail("vh_max_temperature", h, r); break; }
    const double tmax_mev = 1000 * tmax_gev;
    if (!o.quiet) {
      const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
      std::printf("Time Step is %g @  TempMax is %.4f MeV at TAU -->%.4f This is tau step no. %d at time %.5f seconds\n",
                  ts, tmax_mev, tau, l, sec);
    }
    if (std::fabs((tau - tau_print) - o.print_every) < 1e-6) {
      tau_print += o.print_every;
      if ((r = write(tau))) { status = fail("vh_write", h, r); break; }
    }
    if (std::fabs(tau - (c.tau0 + ts)) < 1e-6 && (r = write(tau))) { status = fail("vh_write", h, r); break; }
    l++;
    if (gubser && tau > 9) break;             // main.cpp:196-199
    if (!gubser && !shock && !bjorken && tmax_mev < 120) break;  // main.cpp:201-204
    if (bjorken && tau > 10) break;           // main.cpp:208-210
    if (tau > o.tau_end) break;                // main.cpp:211
    if (o.max_steps > 0 && l > o.max_steps) break;
  }
  if (temp_txt) std::fclose(temp_txt);
  if (!status && !o.checkpoint.empty() && (r = vh_save_checkpoint(h, o.checkpoint.c_str())))
    status = fail("vh_save_checkpoint", h, r);
  double sums[4];
  if (!status && vh_conservation_sums(h, sums) == VH_OK && !o.quiet)
    std::printf("tau %.4f fm/c after %d steps; sum tau T^{tau mu} dV = %.10e %.10e %.10e %.10e\n", tau, l - 1, sums[0],
                sums[1], sums[2], sums[3]);
  vh_destroy(h);
  return status;
}
