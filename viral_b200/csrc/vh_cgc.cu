// The reference's optical-Glauber CGC initial tensor (NEWEST5/ginit.h:658-913),
// host side: nuclear thickness functions, their WENO derivatives and the
// early-time energy-momentum tensor of the classical gluon field to order
// tau^2, on the ghost-inclusive grid.  Landau matching of the result runs on
// the GPU (vh_init_tmunu, vh_init_prevu_tmunu).
#include <cmath>
#include <vector>

#include "vh.h"
#include "vh_device.cuh"

namespace {

// 20-point Gauss-Legendre nodes and weights on [-1, 1]: roots of P_20 by
// Newton's method from the Tricomi estimates
struct GaussLegendre20 {
  double x[20], w[20];
  GaussLegendre20() {
    const int n = 20;
    for (int i = 0; i < n; i++) {
      double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 1;
      for (int it = 0; it < 100; it++) {
        double p0 = 1, p1 = z;
        for (int k = 2; k <= n; k++) {
          const double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
          p0 = p1;
          p1 = p2;
        }
        dp = n * (z * p1 - p0) / (z * z - 1);
        const double step = p1 / dp;
        z -= step;
        if (std::fabs(step) < 1e-16) break;
      }
      x[i] = z;
      w[i] = 2 / ((1 - z * z) * dp * dp);
    }
  }
};

// Woods-Saxon density integrated along the beam axis, 2 s int_0^250 rho dz
// (NEWEST5/ginit.h:44-67, 683-705): rho = rho0 / (1 + exp((r - R)/a)),
// R = 1.12 A^(1/3) - 0.86 A^(-1/3), rho0 = A / (4/3 pi R^3).  Panels of
// width a out to R + 40a carry all but e^-40 of it; 20-point Gauss-Legendre
// per panel integrates the smooth Fermi profile to rounding.
double thickness(const GaussLegendre20& gl, double rho2, double A, double a, double s) {
  const double R = 1.12 * std::cbrt(A) - 0.86 / std::cbrt(A);
  const double rho0 = A / ((4.0 / 3.0) * M_PI * R * R * R);
  const double zmax = std::fmin(250.0, R + 40 * a);
  const int panels = (int)std::ceil(zmax / a);
  const double h = zmax / panels;
  double sum = 0;
  for (int p = 0; p < panels; p++) {
    const double m = (p + 0.5) * h, hh = 0.5 * h;
    double ps = 0;
    for (int q = 0; q < 20; q++) {
      const double z = m + hh * gl.x[q];
      const double r = std::sqrt(rho2 + z * z);
      ps += gl.w[q] * rho0 / (1.0 + std::exp((r - R) / a));
    }
    sum += ps * hh;
  }
  return 2 * s * sum;
}

// the reference's WENO derivative of five samples (NEWEST5/utils.h:57-98)
inline double weno_der(double qm2, double qm1, double qc, double qp1, double qp2, double d) {
  return (vh::weno_left<double>(qm2, qm1, qc, qp1, qp2) - vh::weno_right<double>(qm2, qm1, qc, qp1, qp2)) / d;
}

}  // namespace

extern "C" int vh_profile_cgc(int nx, int ny, int nz, int boost_invariant, double dx, double dy, double dz, double tau,
                              double x_pos, double mass_number, double ws_a, double thickness_scale, double e_peak,
                              double eta_flat, double delta, double* tmunu10) {
  if (nx < 1 || ny < 1 || (!boost_invariant && nz < 1) || !(dx > 0) || !(dy > 0) || !(tau > 0) ||
      !(mass_number > 0) || !(ws_a > 0) || !(e_peak > 0) || !tmunu10)
    return VH_E_ARG;
  const int G = 3, PAD = 18;  // ghost layers; the reference's NOS * BORDER extension
  const int gx = nx + 2 * G, gy = ny + 2 * G, gz = boost_invariant ? 1 : nz + 2 * G;
  const int xt = gx + 2 * PAD, yt = gy + 2 * PAD;
  const size_t nt = (size_t)xt * yt;
  const double x0 = -((double)(nx / 2) * dx), y0 = -((double)(ny / 2) * dy);
  std::vector<double> X(xt), Y(yt);
  for (int i = 0; i < xt; i++) X[i] = x0 + (i - PAD - G) * dx;
  for (int j = 0; j < yt; j++) Y[j] = y0 + (j - PAD - G) * dy;

  // thickness of the nucleus at +x_pos (mu1) and at -x_pos (mu2); the
  // integral depends on the transverse distance only, so equal squared
  // distances share one evaluation
  const GaussLegendre20 gl;
  std::vector<double> mu1(nt), mu2(nt), m12(nt);
  std::vector<std::pair<double, double>> memo;
  auto T_of = [&](double r2) {
    for (const auto& p : memo)
      if (p.first == r2) return p.second;
    const double v = thickness(gl, r2, mass_number, ws_a, thickness_scale);
    memo.emplace_back(r2, v);
    return v;
  };
  std::vector<double> col1(yt), col2(yt);
  double mmax = 0;
  for (int i = 0; i < xt; i++) {
    memo.clear();
    const double d1 = X[i] - x_pos, d2 = X[i] + x_pos;
    for (int j = 0; j < yt; j++) {
      const size_t c = (size_t)i * yt + j;
      mu1[c] = T_of(d1 * d1 + Y[j] * Y[j]);
    }
    memo.clear();
    for (int j = 0; j < yt; j++) {
      const size_t c = (size_t)i * yt + j;
      mu2[c] = T_of(d2 * d2 + Y[j] * Y[j]);
      m12[c] = mu1[c] * mu2[c];
      if (m12[c] > mmax) mmax = m12[c];
    }
  }
  const double norm = e_peak / mmax;

  // derivatives on the extended grid (zero on its two outer layers): of a
  // positive field f as f d(log f) (ginit.h:229-296), of the vectors plainly
  // (ginit.h:161-227)
  auto dx_log = [&](const std::vector<double>& f, std::vector<double>& out) {
    out.assign(nt, 0.0);
    for (int i = 2; i < xt - 2; i++)
      for (int j = 0; j < yt; j++) {
        const size_t c = (size_t)i * yt + j;
        out[c] = f[c] * weno_der(std::log(f[c - 2 * yt]), std::log(f[c - yt]), std::log(f[c]), std::log(f[c + yt]),
                                 std::log(f[c + 2 * yt]), dx);
      }
  };
  auto dy_log = [&](const std::vector<double>& f, std::vector<double>& out) {
    out.assign(nt, 0.0);
    for (int i = 0; i < xt; i++)
      for (int j = 2; j < yt - 2; j++) {
        const size_t c = (size_t)i * yt + j;
        out[c] = f[c] * weno_der(std::log(f[c - 2]), std::log(f[c - 1]), std::log(f[c]), std::log(f[c + 1]),
                                 std::log(f[c + 2]), dy);
      }
  };
  auto dx_plain = [&](const std::vector<double>& f, std::vector<double>& out) {
    out.assign(nt, 0.0);
    for (int i = 2; i < xt - 2; i++)
      for (int j = 0; j < yt; j++) {
        const size_t c = (size_t)i * yt + j;
        out[c] = weno_der(f[c - 2 * yt], f[c - yt], f[c], f[c + yt], f[c + 2 * yt], dx);
      }
  };
  auto dy_plain = [&](const std::vector<double>& f, std::vector<double>& out) {
    out.assign(nt, 0.0);
    for (int i = 0; i < xt; i++)
      for (int j = 2; j < yt - 2; j++) {
        const size_t c = (size_t)i * yt + j;
        out[c] = weno_der(f[c - 2], f[c - 1], f[c], f[c + 1], f[c + 2], dy);
      }
  };
  std::vector<double> dx12, dy12, dx1, dy1, dx2, dy2;
  dx_log(m12, dx12);
  dy_log(m12, dy12);
  dx_log(mu1, dx1);
  dy_log(mu1, dy1);
  dx_log(mu2, dx2);
  dy_log(mu2, dy2);
  // ginit.h:785-792: alpha = -grad(eps), beta = mu1 grad(mu2) - mu2 grad(mu1)
  std::vector<double> ax(nt), ay(nt), bx(nt), by(nt);
  for (size_t c = 0; c < nt; c++) {
    ax[c] = -norm * dx12[c];
    ay[c] = -norm * dy12[c];
    bx[c] = norm * (-dx1[c] * mu2[c] + mu1[c] * dx2[c]);
    by[c] = norm * (-dy1[c] * mu2[c] + mu1[c] * dy2[c]);
  }
  std::vector<double> dxax, dyay, dxbx, dyby;
  dx_plain(ax, dxax);
  dx_plain(bx, dxbx);
  dy_plain(ay, dyay);
  dy_plain(by, dyby);

  // T^{mu nu} per cell (ginit.h:873-905), times the eta cutoff: flat for
  // |eta| < eta_flat/2, Gaussian tails of unit width
  const size_t n = (size_t)gx * gy * gz;
  const double t2 = tau * tau;
  for (int k = 0; k < gz; k++) {
    const double eta = boost_invariant ? 0.0 : -((double)(nz / 2) * dz) + (k - G) * dz;
    const double ae = std::fabs(eta) - 0.5 * eta_flat;
    const double g = ae / std::sqrt(2.0);
    const double cut = std::exp(-g * g * (ae >= 0 ? 1.0 : 0.0));
    for (int j = 0; j < gy; j++)
      for (int i = 0; i < gx; i++) {
        const size_t e = (size_t)(i + PAD) * yt + (j + PAD);
        const double ee = norm * m12[e], dt = delta * ee;
        const double Le = -(dxax[e] + dyay[e]), DB = dxbx[e] + dyby[e];
        double t[10];
        t[0] = ee - 0.125 * t2 * (-2 * Le + dt);  // tt
        t[1] = 0.5 * tau * ax[e];                 // tx
        t[2] = 0.5 * tau * ay[e];                 // ty
        t[3] = 0.125 * tau * DB;                  // t eta
        t[4] = ee - 0.25 * t2 * (-Le + dt);       // xx
        t[5] = 0;                                 // xy
        t[6] = 0.5 * bx[e];                       // x eta
        t[7] = t[4];                              // yy
        t[8] = 0.5 * by[e];                       // y eta
        t[9] = -ee / t2 + 0.125 * (-2 * Le + 3 * dt);  // eta eta
        const size_t c = ((size_t)k * gy + j) * gx + i;
        for (int q = 0; q < 10; q++) tmunu10[q * n + c] = t[q] * cut;
      }
  }
  return VH_OK;
}
