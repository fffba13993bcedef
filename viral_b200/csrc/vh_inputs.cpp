// Seeded host-side input generators (include/vh.h "inputs"): the synthetic
// tabulated EOS, the ideal, cold-plasma and Israel-Stewart Gubser profiles
// and a Monte-Carlo Glauber energy density.  The reference reads its Gubser table from a file it does not
// ship (NEWEST5/init.h:419-459) and builds optical-Glauber/CGC profiles with
// GSL (NEWEST5/ginit.h); these generators stand in for both so that the GPU
// path and its tests consume identical inputs.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "vh.h"

namespace {

// splitmix64 (Steele, Lea, Flood 2014): a small seeded generator
struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
};

double cs2_synth(double e_gev) {
  const double l = std::log(e_gev / 0.5);
  return 1.0 / 3.0 - 0.2 * std::exp(-0.5 * l * l);
}

void axis_coords(int n, int ghost, double d, std::vector<double>& out) {
  out.resize(n + 2 * ghost);
  const double x0 = -((double)(n / 2) * d);
  for (int i = 0; i < n + 2 * ghost; i++) out[i] = x0 + (i - ghost) * d;
}

}  // namespace

extern "C" int vh_eos_table_synthetic(int n, double emin, double emax, double a, double hbarc, double* e,
                                      double* p, double* cs2, double* t) {
  if (n < 2 || !(emin > 0) || !(emax > emin) || !(a > 0) || !(hbarc > 0) || !e || !p || !cs2 || !t) return VH_E_ARG;
  // integrate dP/ds = cs2 e, d lnT/ds = cs2 e/(e+P) in s = ln e with RK4,
  // 32 substeps per row (GeV units), then anchor T(emax) = (emax/a)^(1/4)
  const double s0 = std::log(emin), ds_row = (std::log(emax) - s0) / (n - 1);
  const int sub = 32;
  const double h = ds_row / sub;
  double P = cs2_synth(emin) * emin, lt = 0.0;
  std::vector<double> lts(n);
  auto f = [](double s, double P, double& dP, double& dl) {
    const double ee = std::exp(s), c = cs2_synth(ee);
    dP = c * ee;
    dl = c * ee / (ee + P);
  };
  for (int i = 0; i < n; i++) {
    const double s = s0 + i * ds_row;
    const double ee = std::exp(s);
    e[i] = ee; p[i] = P; cs2[i] = cs2_synth(ee); lts[i] = lt;
    if (i == n - 1) break;
    for (int q = 0; q < sub; q++) {
      const double sq = s + q * h;
      double k1p, k1l, k2p, k2l, k3p, k3l, k4p, k4l;
      f(sq, P, k1p, k1l);
      f(sq + 0.5 * h, P + 0.5 * h * k1p, k2p, k2l);
      f(sq + 0.5 * h, P + 0.5 * h * k2p, k3p, k3l);
      f(sq + h, P + h * k3p, k4p, k4l);
      P += h / 6.0 * (k1p + 2 * k2p + 2 * k3p + k4p);
      lt += h / 6.0 * (k1l + 2 * k2l + 2 * k3l + k4l);
    }
  }
  // to fm units: e, P in fm^-4, T in fm^-1; e = a T^4 holds in fm units
  const double tmax_fm = std::pow(e[n - 1] / hbarc / a, 0.25);
  for (int i = 0; i < n; i++) {
    e[i] /= hbarc;
    p[i] /= hbarc;
    t[i] = tmax_fm * std::exp(lts[i] - lts[n - 1]);
  }
  return VH_OK;
}

extern "C" int vh_profile_gubser(int nx, int ny, double dx, double dy, double q, double tau0, double dtau,
                                 double t0_gev, double a, double hbarc, double* e, double* ux, double* uy,
                                 double* prevu4) {
  if (nx < 1 || ny < 1 || !e || !ux || !uy || !(tau0 > dtau) || !(q > 0)) return VH_E_ARG;
  std::vector<double> X, Y;
  axis_coords(nx, 3, dx, X);
  axis_coords(ny, 3, dy, Y);
  const int gx = nx + 6, gy = ny + 6;
  const long long n = (long long)gx * gy;
  const double q2 = q * q;
  const double t0fm = t0_gev / hbarc;
  // ideal conformal Gubser flow: T ~ tau^(-1/3) [1 + 2q^2(tau^2+r^2) + q^4(tau^2-r^2)^2]^(-1/3),
  // transverse rapidity kappa = atanh(2 q^2 tau r / (1 + q^2 tau^2 + q^2 r^2))
  auto denom = [&](double tau, double r) {
    const double d = tau * tau - r * r;
    return 1 + 2 * q2 * (tau * tau + r * r) + q2 * q2 * d * d;
  };
  const double norm = denom(tau0, 0.0);
  for (int j = 0; j < gy; j++)
    for (int i = 0; i < gx; i++) {
      const long long c = (long long)j * gx + i;
      const double x = X[i], y = Y[j], r = std::sqrt(x * x + y * y);
      const double T = t0fm * std::cbrt(norm / denom(tau0, r));
      e[c] = a * T * T * T * T;
      for (int pass = 0; pass < 2; pass++) {
        const double tau = pass ? tau0 - dtau : tau0;
        const double k = std::atanh(2 * q2 * tau * r / (1 + q2 * tau * tau + q2 * r * r));
        const double sh = std::sinh(k), ch = std::cosh(k);
        const double vx = r > 0 ? sh * x / r : 0.0, vy = r > 0 ? sh * y / r : 0.0;
        if (!pass) { ux[c] = vx; uy[c] = vy; }
        else if (prevu4) {
          prevu4[c] = ch; prevu4[n + c] = vx; prevu4[2 * n + c] = vy; prevu4[3 * n + c] = 0.0;
        }
      }
    }
  return VH_OK;
}

extern "C" int vh_profile_gubser_cold(int nx, int ny, double dx, double dy, double q, double tau0, double dtau,
                                      double b, double a, double* e, double* ux, double* uy, double* pi5,
                                      double* prevu4) {
  if (nx < 1 || ny < 1 || !e || !ux || !uy || !pi5 || !(tau0 > dtau) || !(q > 0) || !(b > 0) || !(a > 0))
    return VH_E_ARG;
  std::vector<double> X, Y;
  axis_coords(nx, 3, dx, X);
  axis_coords(ny, 3, dy, Y);
  const int gx = nx + 6, gy = ny + 6;
  const long long n = (long long)gx * gy;
  const double q2 = q * q, k = 4.0 / (3.0 * std::sqrt(5.0));
  for (int j = 0; j < gy; j++)
    for (int i = 0; i < gx; i++) {
      const long long c = (long long)j * gx + i;
      const double x = X[i], y = Y[j], r = std::sqrt(x * x + y * y);
      for (int pass = 0; pass < 2; pass++) {
        const double tau = pass ? tau0 - dtau : tau0;
        const double kap = std::atanh(2 * q2 * tau * r / (1 + q2 * tau * tau + q2 * r * r));
        const double sh = std::sinh(kap), ch = std::cosh(kap);
        const double cphi = r > 0 ? x / r : 1.0, sphi = r > 0 ? y / r : 0.0;
        if (pass) {
          if (prevu4) {
            prevu4[c] = ch; prevu4[n + c] = sh * cphi; prevu4[2 * n + c] = sh * sphi; prevu4[3 * n + c] = 0.0;
          }
          continue;
        }
        ux[c] = sh * cphi;
        uy[c] = sh * sphi;
        // de Sitter time rho and the cold-plasma solution there: the shear
        // ratio pi^eta_eta / (e + P) relaxes nowhere and follows
        // d(pibar)/d(ln cosh rho) = 4/15 - (4/3) pibar^2 from 0 at rho = 0
        const double rho = std::asinh(-(1 - q2 * tau * tau + q2 * r * r) / (2 * q * tau));
        const double lc = std::log(std::cosh(rho));
        const double That = b * std::pow(std::cosh(k * lc), 0.25) / std::pow(std::cosh(rho), 2.0 / 3.0);
        const double T = That / tau;
        e[c] = a * T * T * T * T;
        const double w_hat = (4.0 / 3.0) * a * That * That * That * That;
        const double pihat = -w_hat * std::tanh(k * lc) / std::sqrt(5.0);
        // Milne: the eta and phi directions carry pihat / tau^4 (mixed
        // components, pi^theta_theta = pi^phi_phi = -pihat/2); the direction
        // in the (tau, r) plane orthogonal to u, n = (sinh kap, cosh kap),
        // carries pi^{ab} = (pihat / (2 tau^4)) n^a n^b
        const double c0 = pihat / (2 * tau * tau * tau * tau);
        const double prr = c0 * ch * ch, pff = c0;  // pi^{rr}, r^2 pi^{phi phi}
        pi5[c] = cphi * cphi * prr + sphi * sphi * pff;          // xx
        pi5[n + c] = sphi * sphi * prr + cphi * cphi * pff;      // yy
        pi5[2 * n + c] = sphi * cphi * (prr - pff);              // xy
        pi5[3 * n + c] = 0.0;                                    // x eta
        pi5[4 * n + c] = 0.0;                                    // y eta
      }
    }
  return VH_OK;
}

namespace {

// The Israel-Stewart Gubser flow (conformal fluid, tau_pi = 5 eta/(e+P),
// constant eta/s) as functions of the de Sitter time rho, sinh rho =
// -(1 - q^2 tau^2 + q^2 r^2)/(2 q tau): T^ = tau T and the shear ratio
// P = tau^2 pi^{eta eta}/(e + P_pressure), both Weyl invariant.  In the
// fluid's rest frame of de Sitter space (theta^ = 2 tanh rho,
// sigma^{eta eta} = (2/3) tanh rho in the reference's mostly-minus
// convention) energy conservation and the relaxation equation
// tau_pi (D pi + (4/3) pi theta) + pi = 2 eta sigma become
//   d ln T^/d rho = -(2/3) tanh rho + (1/3) P tanh rho
//   dP/d rho      = -(4/3) P^2 tanh rho - P T^/(5 eta/s) + (4/15) tanh rho.
// Integrated by classical RK4 on a uniform rho grid outward from rho0 in
// both directions; values between nodes by cubic Hermite interpolation with
// the right-hand side as the derivative.
struct GubserIS {
  double etas, rho0, h;
  std::vector<double> lt, pb;  // node values from rho_lo upward
  double rho_lo = 0;

  void rhs(double rho, double l, double p, double& dl, double& dp) const {
    const double th = std::tanh(rho), T = std::exp(l);
    dl = -(2.0 / 3.0) * th + (1.0 / 3.0) * p * th;
    dp = -(4.0 / 3.0) * p * p * th - p * T / (5.0 * etas) + (4.0 / 15.0) * th;
  }
  // n steps of size hs (signed) from (rho, l, p), appending the nodes
  void march(double rho, double l, double p, double hs, int n, std::vector<double>& L, std::vector<double>& Pv) const {
    for (int i = 0; i < n; i++) {
      double k1l, k1p, k2l, k2p, k3l, k3p, k4l, k4p;
      rhs(rho, l, p, k1l, k1p);
      rhs(rho + 0.5 * hs, l + 0.5 * hs * k1l, p + 0.5 * hs * k1p, k2l, k2p);
      rhs(rho + 0.5 * hs, l + 0.5 * hs * k2l, p + 0.5 * hs * k2p, k3l, k3p);
      rhs(rho + hs, l + hs * k3l, p + hs * k3p, k4l, k4p);
      l += hs / 6.0 * (k1l + 2 * k2l + 2 * k3l + k4l);
      p += hs / 6.0 * (k1p + 2 * k2p + 2 * k3p + k4p);
      rho += hs;
      L.push_back(l);
      Pv.push_back(p);
    }
  }
  bool build(double t_hat0, double p0, double lo, double hi) {
    if (!(t_hat0 > 0) || !(etas > 0) || lo > rho0 || hi < rho0) return false;
    const int nd = (int)std::ceil((rho0 - lo) / h) + 2, nu = (int)std::ceil((hi - rho0) / h) + 2;
    std::vector<double> Ld, Pd, Lu, Pu;
    march(rho0, std::log(t_hat0), p0, -h, nd, Ld, Pd);
    march(rho0, std::log(t_hat0), p0, h, nu, Lu, Pu);
    lt.assign(Ld.rbegin(), Ld.rend());
    pb.assign(Pd.rbegin(), Pd.rend());
    lt.push_back(std::log(t_hat0));
    pb.push_back(p0);
    lt.insert(lt.end(), Lu.begin(), Lu.end());
    pb.insert(pb.end(), Pu.begin(), Pu.end());
    rho_lo = rho0 - nd * h;
    for (size_t i = 0; i < lt.size(); i++)
      if (!std::isfinite(lt[i]) || !std::isfinite(pb[i])) return false;
    return true;
  }
  void at(double rho, double& t_hat, double& p) const {
    const double u = (rho - rho_lo) / h;
    int i = (int)std::floor(u);
    i = i < 0 ? 0 : (i > (int)lt.size() - 2 ? (int)lt.size() - 2 : i);
    const double s = u - i, r0 = rho_lo + i * h;
    double d0l, d0p, d1l, d1p;
    rhs(r0, lt[i], pb[i], d0l, d0p);
    rhs(r0 + h, lt[i + 1], pb[i + 1], d1l, d1p);
    const double h00 = (1 + 2 * s) * (1 - s) * (1 - s), h10 = s * (1 - s) * (1 - s), h01 = s * s * (3 - 2 * s),
                 h11 = s * s * (s - 1);
    const double l = h00 * lt[i] + h10 * h * d0l + h01 * lt[i + 1] + h11 * h * d1l;
    p = h00 * pb[i] + h10 * h * d0p + h01 * pb[i + 1] + h11 * h * d1p;
    t_hat = std::exp(l);
  }
};

}  // namespace

extern "C" int vh_profile_gubser_is(int nx, int ny, double dx, double dy, double q, double tau0, double dtau,
                                    double t0_gev, double p0, double etas, double a, double hbarc, double* e,
                                    double* ux, double* uy, double* pi5, double* prevu4) {
  if (nx < 1 || ny < 1 || !e || !ux || !uy || !pi5 || !(tau0 > dtau) || !(q > 0) || !(etas > 0) || !(a > 0) ||
      !(hbarc > 0) || !(t0_gev > 0))
    return VH_E_ARG;
  std::vector<double> X, Y;
  axis_coords(nx, 3, dx, X);
  axis_coords(ny, 3, dy, Y);
  const int gx = nx + 6, gy = ny + 6;
  const long long n = (long long)gx * gy;
  const double q2 = q * q;
  auto rho_of = [&](double tau, double r) { return std::asinh(-(1 - q2 * tau * tau + q2 * r * r) / (2 * q * tau)); };
  // the solution is fixed at the grid centre at tau0: T^ = tau0 T0, P = p0
  GubserIS G{etas, rho_of(tau0, 0.0), 1e-3, {}, {}};
  double rmax = 0;
  for (double x : X)
    for (double y : Y) rmax = std::max(rmax, std::sqrt(x * x + y * y));
  if (!G.build(tau0 * t0_gev / hbarc, p0, rho_of(tau0, rmax) - 0.01, G.rho0 + 0.01)) return VH_E_ARG;
  for (int j = 0; j < gy; j++)
    for (int i = 0; i < gx; i++) {
      const long long c = (long long)j * gx + i;
      const double x = X[i], y = Y[j], r = std::sqrt(x * x + y * y);
      const double cphi = r > 0 ? x / r : 1.0, sphi = r > 0 ? y / r : 0.0;
      for (int pass = 0; pass < 2; pass++) {
        const double tau = pass ? tau0 - dtau : tau0;
        const double kap = std::atanh(2 * q2 * tau * r / (1 + q2 * tau * tau + q2 * r * r));
        const double sh = std::sinh(kap), ch = std::cosh(kap);
        if (pass) {
          if (prevu4) {
            prevu4[c] = ch; prevu4[n + c] = sh * cphi; prevu4[2 * n + c] = sh * sphi; prevu4[3 * n + c] = 0.0;
          }
          continue;
        }
        ux[c] = sh * cphi;
        uy[c] = sh * sphi;
        double t_hat, pr;
        G.at(rho_of(tau, r), t_hat, pr);
        const double T = t_hat / tau;
        e[c] = a * T * T * T * T;
        // rest-frame shear: w P along eta (orthonormal), -w P/2 along phi and
        // along n = (sinh kap, cosh kap cos phi, cosh kap sin phi), the unit
        // vector of the (tau, r) plane orthogonal to u
        const double w = (4.0 / 3.0) * e[c], hp = -0.5 * w * pr;
        pi5[c] = hp * (sphi * sphi + ch * ch * cphi * cphi);          // xx
        pi5[n + c] = hp * (cphi * cphi + ch * ch * sphi * sphi);      // yy
        pi5[2 * n + c] = hp * sphi * cphi * (ch * ch - 1.0);          // xy
        pi5[3 * n + c] = 0.0;                                         // x eta
        pi5[4 * n + c] = 0.0;                                         // y eta
      }
    }
  return VH_OK;
}

extern "C" int vh_profile_glauber(int nx, int ny, int nz, int boost_invariant, double dx, double dy, double dz, int A,
                                  double R, double aws, double dmin, double b, double sigma_nn, double w,
                                  double epeak_gev, double eta_flat, double eta_sigma, double efloor_gev,
                                  double hbarc, uint64_t seed, double* e, int* npart) {
  if (nx < 1 || ny < 1 || A < 1 || !e || !(w > 0) || !(sigma_nn > 0) || !(epeak_gev > 0)) return VH_E_ARG;
  Rng rng(seed * 0x9E3779B97F4A7C15ull + 12345);
  // nucleon positions: radius from r^2 / (1 + exp((r-R)/a)) by rejection,
  // isotropic direction, no two nucleons of a nucleus closer than dmin
  const double rmax = R + 10 * aws;
  auto sample_nucleus = [&](double xc, std::vector<double>& xs, std::vector<double>& ys) {
    std::vector<double> px, py, pz;
    int placed = 0;
    while (placed < A) {
      double r;
      for (;;) {
        r = rmax * rng.uniform();
        const double acc = (r / rmax) * (r / rmax) / (1.0 + std::exp((r - R) / aws));
        if (rng.uniform() < acc) break;
      }
      const double ct = 2 * rng.uniform() - 1, st = std::sqrt(std::max(0.0, 1 - ct * ct));
      const double ph = 2 * M_PI * rng.uniform();
      const double x = r * st * std::cos(ph), y = r * st * std::sin(ph), z = r * ct;
      bool ok = true;
      for (int q = 0; q < placed && ok; q++) {
        const double ddx = px[q] - x, ddy = py[q] - y, ddz = pz[q] - z;
        if (ddx * ddx + ddy * ddy + ddz * ddz < dmin * dmin) ok = false;
      }
      if (!ok) continue;
      px.push_back(x); py.push_back(y); pz.push_back(z);
      placed++;
    }
    xs.resize(A); ys.resize(A);
    for (int q = 0; q < A; q++) { xs[q] = px[q] + xc; ys[q] = py[q]; }
  };
  std::vector<double> ax, ay, bx, by;
  sample_nucleus(-0.5 * b, ax, ay);
  sample_nucleus(+0.5 * b, bx, by);
  const double d2 = sigma_nn / M_PI;
  std::vector<char> pa(A, 0), pb(A, 0);
  for (int i = 0; i < A; i++)
    for (int j = 0; j < A; j++) {
      const double ddx = ax[i] - bx[j], ddy = ay[i] - by[j];
      if (ddx * ddx + ddy * ddy <= d2) { pa[i] = 1; pb[j] = 1; }
    }
  std::vector<double> sx, sy;
  for (int i = 0; i < A; i++) if (pa[i]) { sx.push_back(ax[i]); sy.push_back(ay[i]); }
  for (int j = 0; j < A; j++) if (pb[j]) { sx.push_back(bx[j]); sy.push_back(by[j]); }
  if (npart) *npart = (int)sx.size();
  std::vector<double> X, Y, Z;
  axis_coords(nx, 3, dx, X);
  axis_coords(ny, 3, dy, Y);
  const int gx = nx + 6, gy = ny + 6, gz = boost_invariant ? 1 : nz + 6;
  if (boost_invariant) Z.assign(1, 0.0); else axis_coords(nz, 3, dz, Z);
  std::vector<double> et((size_t)gx * gy, 0.0);
  const double i2w2 = 1.0 / (2 * w * w);
  double emax = 0;
  for (int j = 0; j < gy; j++)
    for (int i = 0; i < gx; i++) {
      double s = 0;
      for (size_t q = 0; q < sx.size(); q++) {
        const double ddx = X[i] - sx[q], ddy = Y[j] - sy[q];
        s += std::exp(-(ddx * ddx + ddy * ddy) * i2w2);
      }
      et[(size_t)j * gx + i] = s;
      if (i >= 3 && i < 3 + nx && j >= 3 && j < 3 + ny) emax = std::max(emax, s);
    }
  // peak e over the interior is epeak; the floor keeps pressure and
  // temperature positive far outside the fireball
  const double scale = emax > 0 ? epeak_gev / hbarc / emax : 0.0;
  const double floor_fm = efloor_gev / hbarc;
  for (int k = 0; k < gz; k++) {
    const double ae = std::fabs(Z[k]);
    const double fz = ae <= eta_flat ? 1.0 : std::exp(-0.5 * (ae - eta_flat) * (ae - eta_flat) / (eta_sigma * eta_sigma));
    for (int j = 0; j < gy; j++)
      for (int i = 0; i < gx; i++) {
        const double v = et[(size_t)j * gx + i] * scale * fz;
        e[((size_t)k * gy + j) * gx + i] = v > floor_fm ? v : floor_fm;
      }
  }
  return VH_OK;
}
