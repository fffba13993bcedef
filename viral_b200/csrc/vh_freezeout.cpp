// Isothermal freeze-out hypersurface and Boltzmann Cooper-Frye spectra,
// host entry points: the per-cube arithmetic of vh_freezeout.cuh run over
// the grid in cube order (x fastest), the order in which the device kernels
// of vh_freezeout_dev.cu also emit.  The reference stops at the freeze-out
// temperature (NEWEST5/main.cpp:201-204, MaxTempGev in utils.h:263) and has
// no hypersurface; this is the step after the path.
#include <cmath>

#include "vh.h"
#include "vh_freezeout.cuh"

extern "C" int vh_freezeout_2d(int nx, int ny, double dx, double dy, double tau0, double tau1, const double* t0,
                               const double* t1, const double* u0, const double* u1, double t_fo, double* out,
                               long long cap, long long* count) {
  if (nx < 2 || ny < 2 || !(dx > 0) || !(dy > 0) || !(tau1 > tau0) || !t0 || !t1 || !u0 || !u1 || !count ||
      (cap > 0 && !out) || cap < 0)
    return VH_E_ARG;
  const vh_fo::Geo g = vh_fo::make_geo(nx, ny, 1, dx, dy, 0.0, tau0, tau1, t_fo, true);
  vh_fo::Sink s{out, 0, cap};
  for (int j = vh_fo::kG; j < vh_fo::kG + ny - 1; j++)
    for (int i = vh_fo::kG; i < vh_fo::kG + nx - 1; i++) vh_fo::cube2(g, i, j, t0, t1, u0, u1, s);
  *count = s.at;
  return s.at > cap ? VH_E_ARG : VH_OK;
}

extern "C" int vh_freezeout_3d(int nx, int ny, int nz, double dx, double dy, double dz, double tau0, double tau1,
                               const double* t0, const double* t1, const double* u0, const double* u1, double t_fo,
                               double* out, long long cap, long long* count) {
  if (nx < 2 || ny < 2 || nz < 2 || !(dx > 0) || !(dy > 0) || !(dz > 0) || !(tau1 > tau0) || !t0 || !t1 || !u0 ||
      !u1 || !count || (cap > 0 && !out) || cap < 0)
    return VH_E_ARG;
  const vh_fo::Geo g = vh_fo::make_geo(nx, ny, nz, dx, dy, dz, tau0, tau1, t_fo, false);
  vh_fo::Sink s{out, 0, cap};
  for (int k = vh_fo::kG; k < vh_fo::kG + nz - 1; k++)
    for (int j = vh_fo::kG; j < vh_fo::kG + ny - 1; j++)
      for (int i = vh_fo::kG; i < vh_fo::kG + nx - 1; i++) vh_fo::cube3(g, i, j, k, t0, t1, u0, u1, s);
  *count = s.at;
  return s.at > cap ? VH_E_ARG : VH_OK;
}

// ------------------------------------------------------ Cooper-Frye spectra
// Boltzmann spectrum at mid-rapidity from the surface elements of
// vh_freezeout_2d (boost invariant, u^eta = 0): with p^mu dSigma_mu =
// m_T cosh(y - eta) dSigma_tau + p_x dSigma_x + p_y dSigma_y and
// p.u = m_T u^tau cosh(y - eta) - p_x u^x - p_y u^y, the rapidity integral
// gives Bessel functions, int deta cosh(eta) e^{-a cosh eta} = 2 K1(a) and
// int deta e^{-a cosh eta} = 2 K0(a):
//   E dN/d^3p = g / (2 pi)^3 sum [2 m_T K1(a) dSigma_tau + 2 K0(a) (p_x dSigma_x
//               + p_y dSigma_y)] exp((p_x u^x + p_y u^y) / T),  a = m_T u^tau / T,
// with e^a K0(a), e^a K1(a) by the quadrature of vh_freezeout.cuh and the
// exponentials combined, so that neither factor overflows at large p_T.
extern "C" int vh_cooper_frye_2d(const double* elements, long long count, double t_fo, double mass, double degeneracy,
                                 const double* pt, int npt, const double* phi, int nphi, double* out) {
  if (!elements || count < 0 || !(t_fo > 0) || !(mass >= 0) || !pt || !phi || npt < 1 || nphi < 1 || !out ||
      !vh_fo::bins_ok(mass, pt, npt, phi, nphi, false))
    return VH_E_ARG;
  const double pref = degeneracy / (8 * M_PI * M_PI * M_PI);
  for (int a = 0; a < npt; a++)
    for (int b = 0; b < nphi; b++) {
      const double mt = std::sqrt(mass * mass + pt[a] * pt[a]);
      const double px = pt[a] * std::cos(phi[b]), py = pt[a] * std::sin(phi[b]);
      double sum = 0;
      for (long long e = 0; e < count; e++) sum += vh_fo::cf2_term(elements + 9 * e, mt, px, py, t_fo);
      out[(long long)a * nphi + b] = pref * sum;
    }
  return VH_OK;
}

// The same on the 3+1D surface of vh_freezeout_3d, at rapidity y: each
// element sits at its own eta, so the sum runs over the elements directly,
//   p^tau = m_T cosh(y - eta), p^eta = m_T sinh(y - eta) / tau,
//   p.u = p^tau u^tau - p_x u^x - p_y u^y - tau^2 p^eta u^eta,
//   E dN/d^3p = g / (2 pi)^3 sum p^mu dSigma_mu exp(-p.u / T).
extern "C" int vh_cooper_frye_3d(const double* elements, long long count, double t_fo, double mass, double degeneracy,
                                 double y, const double* pt, int npt, const double* phi, int nphi, double* out) {
  if (!elements || count < 0 || !(t_fo > 0) || !(mass >= 0) || !pt || !phi || npt < 1 || nphi < 1 || !out ||
      !vh_fo::bins_ok(mass, pt, npt, phi, nphi, true))
    return VH_E_ARG;
  const double pref = degeneracy / (8 * M_PI * M_PI * M_PI);
  for (int a = 0; a < npt; a++)
    for (int b = 0; b < nphi; b++) {
      const double mt = std::sqrt(mass * mass + pt[a] * pt[a]);
      const double px = pt[a] * std::cos(phi[b]), py = pt[a] * std::sin(phi[b]);
      double sum = 0;
      for (long long e = 0; e < count; e++) sum += vh_fo::cf3_term(elements + 12 * e, mt, px, py, y, t_fo);
      out[(long long)a * nphi + b] = pref * sum;
    }
  return VH_OK;
}
