// Isothermal freeze-out hypersurface of a boost-invariant run, host side:
// the surface T = T_fo between two consecutive time slices of the
// ghost-inclusive grid, as triangles of the linear interpolant in
// (tau, x, y) found by marching tetrahedra (each space-time cube between
// neighbouring cell centres split into six tetrahedra around its diagonal).
// The reference stops at the freeze-out temperature (NEWEST5/main.cpp:201-204,
// MaxTempGev in utils.h:263) and has no hypersurface; this is the step after
// the path.
#include <algorithm>
#include <cmath>
#include <vector>

#include "vh.h"

namespace {

struct Pt {
  double x[3];  // tau, x, y
  double u[3];  // u^tau, u^x, u^y
};

// the six tetrahedra of the unit cube around its diagonal: vertex bits
// (tau, x, y) in the order 0 -> e_a -> e_a + e_b -> (1, 1, 1)
const int kTets[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7}, {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};

struct Emit {
  double* out;
  long long cap, count;
  void triangle(const Pt& a, const Pt& b, const Pt& c, const double* cold, const double* hot) {
    // dSigma_mu = (tau / 2) eps_{mu nu lambda} (b - a)^nu (c - a)^lambda per
    // unit rapidity, oriented from the hot side to the cold side
    double e1[3], e2[3], n[3];
    for (int q = 0; q < 3; q++) { e1[q] = b.x[q] - a.x[q]; e2[q] = c.x[q] - a.x[q]; }
    n[0] = 0.5 * (e1[1] * e2[2] - e1[2] * e2[1]);
    n[1] = 0.5 * (e1[2] * e2[0] - e1[0] * e2[2]);
    n[2] = 0.5 * (e1[0] * e2[1] - e1[1] * e2[0]);
    double d = 0;
    for (int q = 0; q < 3; q++) d += n[q] * (cold[q] - hot[q]);
    const double s = d < 0 ? -1.0 : 1.0;
    const double tc = (a.x[0] + b.x[0] + c.x[0]) / 3;
    if (count < cap) {
      double* o = out + 9 * count;
      for (int q = 0; q < 3; q++) o[q] = (a.x[q] + b.x[q] + c.x[q]) / 3;
      for (int q = 0; q < 3; q++) o[3 + q] = s * tc * n[q];
      for (int q = 0; q < 3; q++) o[6 + q] = (a.u[q] + b.u[q] + c.u[q]) / 3;
    }
    count++;
  }
};

Pt edge_point(const double* xa, const double* xb, const double* ua, const double* ub, double fa, double fb) {
  const double w = fa / (fa - fb);
  Pt p;
  for (int q = 0; q < 3; q++) {
    p.x[q] = xa[q] + w * (xb[q] - xa[q]);
    p.u[q] = ua[q] + w * (ub[q] - ua[q]);
  }
  return p;
}

}  // namespace

extern "C" int vh_freezeout_2d(int nx, int ny, double dx, double dy, double tau0, double tau1, const double* t0,
                               const double* t1, const double* u0, const double* u1, double t_fo, double* out,
                               long long cap, long long* count) {
  if (nx < 2 || ny < 2 || !(dx > 0) || !(dy > 0) || !(tau1 > tau0) || !t0 || !t1 || !u0 || !u1 || !count ||
      (cap > 0 && !out) || cap < 0)
    return VH_E_ARG;
  const int G = 3, gx = nx + 2 * G, gy = ny + 2 * G;
  const long long n = (long long)gx * gy;
  const double x0 = -((double)(nx / 2) * dx), y0 = -((double)(ny / 2) * dy);
  Emit em{out, cap, 0};
  for (int j = G; j < G + ny - 1; j++)
    for (int i = G; i < G + nx - 1; i++) {
      double xs[8][3], us[8][3], f[8];
      bool pos = false, neg = false;
      for (int v = 0; v < 8; v++) {
        const int bt = v & 1, bx = (v >> 1) & 1, by = (v >> 2) & 1;
        const long long c = (long long)(j + by) * gx + (i + bx);
        const double* T = bt ? t1 : t0;
        const double* U = bt ? u1 : u0;
        xs[v][0] = bt ? tau1 : tau0;
        xs[v][1] = x0 + (i + bx - G) * dx;
        xs[v][2] = y0 + (j + by - G) * dy;
        for (int q = 0; q < 3; q++) us[v][q] = U[q * n + c];
        f[v] = T[c] - t_fo;
        if (f[v] > 0) pos = true; else neg = true;
      }
      if (!pos || !neg) continue;
      for (const auto& tet : kTets) {
        int hot[4], cold[4], nh = 0, nc = 0;
        for (int q = 0; q < 4; q++) {
          if (f[tet[q]] > 0) hot[nh++] = tet[q]; else cold[nc++] = tet[q];
        }
        if (!nh || !nc) continue;
        const double* ph = xs[hot[0]];
        const double* pc = xs[cold[0]];
        auto P = [&](int a, int b) { return edge_point(xs[a], xs[b], us[a], us[b], f[a], f[b]); };
        if (nh == 1 || nc == 1) {
          const int lone = nh == 1 ? hot[0] : cold[0];
          const int* other = nh == 1 ? cold : hot;
          em.triangle(P(lone, other[0]), P(lone, other[1]), P(lone, other[2]), pc, ph);
        } else {
          // two against two: a quadrilateral a-b-c-d split into two triangles
          const Pt a = P(hot[0], cold[0]), b = P(hot[0], cold[1]), c = P(hot[1], cold[1]), d = P(hot[1], cold[0]);
          em.triangle(a, b, c, pc, ph);
          em.triangle(a, c, d, pc, ph);
        }
      }
    }
  *count = em.count;
  return em.count > cap ? VH_E_ARG : VH_OK;
}

// ---------------------------------------------------------------- 3+1D
namespace {

struct Pt4 {
  double x[4];  // tau, x, y, eta
  double u[4];
};

// the 24 simplices of the unit 4-cube around its diagonal: one per order of
// the axes, the path 0 -> e_a -> e_a + e_b -> e_a + e_b + e_c -> 15
struct Kuhn4 {
  int s[24][5];
  Kuhn4() {
    int perm[4] = {0, 1, 2, 3}, k = 0;
    do {
      int v = 0;
      s[k][0] = 0;
      for (int q = 0; q < 4; q++) { v |= 1 << perm[q]; s[k][q + 1] = v; }
      k++;
    } while (std::next_permutation(perm, perm + 4));
  }
};

struct Emit4 {
  double* out;
  long long cap, count;
  // dSigma_mu = (tau / 6) eps_{mu nu lambda rho} e1^nu e2^lambda e3^rho for
  // the tetrahedron (a, b, c, d), oriented from the hot side to the cold side
  void tetra(const Pt4& a, const Pt4& b, const Pt4& c, const Pt4& d, const double* cold, const double* hot) {
    double e[3][4];
    for (int q = 0; q < 4; q++) { e[0][q] = b.x[q] - a.x[q]; e[1][q] = c.x[q] - a.x[q]; e[2][q] = d.x[q] - a.x[q]; }
    double n[4];
    for (int m = 0; m < 4; m++) {
      // cofactor of column m of the 4x4 matrix [unit_m; e1; e2; e3]
      int cols[3], k = 0;
      for (int q = 0; q < 4; q++) if (q != m) cols[k++] = q;
      const double det = e[0][cols[0]] * (e[1][cols[1]] * e[2][cols[2]] - e[1][cols[2]] * e[2][cols[1]]) -
                         e[0][cols[1]] * (e[1][cols[0]] * e[2][cols[2]] - e[1][cols[2]] * e[2][cols[0]]) +
                         e[0][cols[2]] * (e[1][cols[0]] * e[2][cols[1]] - e[1][cols[1]] * e[2][cols[0]]);
      n[m] = ((m & 1) ? -det : det) / 6.0;
    }
    double dd = 0;
    for (int q = 0; q < 4; q++) dd += n[q] * (cold[q] - hot[q]);
    const double sg = dd < 0 ? -1.0 : 1.0;
    const double tc = (a.x[0] + b.x[0] + c.x[0] + d.x[0]) / 4;
    if (count < cap) {
      double* o = out + 12 * count;
      for (int q = 0; q < 4; q++) o[q] = (a.x[q] + b.x[q] + c.x[q] + d.x[q]) / 4;
      for (int q = 0; q < 4; q++) o[4 + q] = sg * tc * n[q];
      for (int q = 0; q < 4; q++) o[8 + q] = (a.u[q] + b.u[q] + c.u[q] + d.u[q]) / 4;
    }
    count++;
  }
};

}  // namespace

extern "C" int vh_freezeout_3d(int nx, int ny, int nz, double dx, double dy, double dz, double tau0, double tau1,
                               const double* t0, const double* t1, const double* u0, const double* u1, double t_fo,
                               double* out, long long cap, long long* count) {
  if (nx < 2 || ny < 2 || nz < 2 || !(dx > 0) || !(dy > 0) || !(dz > 0) || !(tau1 > tau0) || !t0 || !t1 || !u0 ||
      !u1 || !count || (cap > 0 && !out) || cap < 0)
    return VH_E_ARG;
  static const Kuhn4 K;
  const int G = 3, gx = nx + 2 * G, gy = ny + 2 * G, gz = nz + 2 * G;
  const long long n = (long long)gx * gy * gz;
  const double x0 = -((double)(nx / 2) * dx), y0 = -((double)(ny / 2) * dy), z0 = -((double)(nz / 2) * dz);
  Emit4 em{out, cap, 0};
  for (int k = G; k < G + nz - 1; k++)
    for (int j = G; j < G + ny - 1; j++)
      for (int i = G; i < G + nx - 1; i++) {
        double xs[16][4], us[16][4], f[16];
        bool pos = false, neg = false;
        for (int v = 0; v < 16; v++) {
          const int bt = v & 1, bx = (v >> 1) & 1, by = (v >> 2) & 1, bz = (v >> 3) & 1;
          const long long c = ((long long)(k + bz) * gy + (j + by)) * gx + (i + bx);
          const double* T = bt ? t1 : t0;
          const double* U = bt ? u1 : u0;
          xs[v][0] = bt ? tau1 : tau0;
          xs[v][1] = x0 + (i + bx - G) * dx;
          xs[v][2] = y0 + (j + by - G) * dy;
          xs[v][3] = z0 + (k + bz - G) * dz;
          for (int q = 0; q < 4; q++) us[v][q] = U[q * n + c];
          f[v] = T[c] - t_fo;
          if (f[v] > 0) pos = true; else neg = true;
        }
        if (!pos || !neg) continue;
        auto P = [&](int a, int b) {
          const double w = f[a] / (f[a] - f[b]);
          Pt4 p;
          for (int q = 0; q < 4; q++) {
            p.x[q] = xs[a][q] + w * (xs[b][q] - xs[a][q]);
            p.u[q] = us[a][q] + w * (us[b][q] - us[a][q]);
          }
          return p;
        };
        for (const auto& sx : K.s) {
          int hot[5], cold[5], nh = 0, nc = 0;
          for (int q = 0; q < 5; q++) {
            if (f[sx[q]] > 0) hot[nh++] = sx[q]; else cold[nc++] = sx[q];
          }
          if (!nh || !nc) continue;
          const double* ph = xs[hot[0]];
          const double* pc = xs[cold[0]];
          if (nh == 1 || nc == 1) {
            // one vertex against four: a tetrahedron
            const int lone = nh == 1 ? hot[0] : cold[0];
            const int* o = nh == 1 ? cold : hot;
            em.tetra(P(lone, o[0]), P(lone, o[1]), P(lone, o[2]), P(lone, o[3]), pc, ph);
          } else {
            // two against three: a triangular prism, as three tetrahedra
            const int* two = nh == 2 ? hot : cold;
            const int* three = nh == 2 ? cold : hot;
            const Pt4 a0 = P(two[0], three[0]), a1 = P(two[0], three[1]), a2 = P(two[0], three[2]);
            const Pt4 b0 = P(two[1], three[0]), b1 = P(two[1], three[1]), b2 = P(two[1], three[2]);
            em.tetra(a0, a1, a2, b0, pc, ph);
            em.tetra(a1, a2, b0, b1, pc, ph);
            em.tetra(a2, b0, b1, b2, pc, ph);
          }
        }
      }
  *count = em.count;
  return em.count > cap ? VH_E_ARG : VH_OK;
}

// ------------------------------------------------------ Cooper-Frye spectra
// Boltzmann spectrum at mid-rapidity from the surface elements of
// vh_freezeout_2d (boost invariant, u^eta = 0): with p^mu dSigma_mu =
// m_T cosh(y - eta) dSigma_tau + p_x dSigma_x + p_y dSigma_y and
// p.u = m_T u^tau cosh(y - eta) - p_x u^x - p_y u^y, the rapidity integral
// gives Bessel functions, int deta cosh(eta) e^{-a cosh eta} = 2 K1(a) and
// int deta e^{-a cosh eta} = 2 K0(a):
//   E dN/d^3p = g / (2 pi)^3 sum [2 m_T K1(a) dSigma_tau + 2 K0(a) (p_x dSigma_x
//               + p_y dSigma_y)] exp((p_x u^x + p_y u^y) / T),  a = m_T u^tau / T.
extern "C" int vh_cooper_frye_2d(const double* elements, long long count, double t_fo, double mass, double degeneracy,
                                 const double* pt, int npt, const double* phi, int nphi, double* out) {
  if (!elements || count < 0 || !(t_fo > 0) || mass < 0 || !pt || !phi || npt < 1 || nphi < 1 || !out)
    return VH_E_ARG;
  const double pref = degeneracy / (8 * M_PI * M_PI * M_PI);
  for (int a = 0; a < npt; a++)
    for (int b = 0; b < nphi; b++) {
      const double mt = std::sqrt(mass * mass + pt[a] * pt[a]);
      const double px = pt[a] * std::cos(phi[b]), py = pt[a] * std::sin(phi[b]);
      double sum = 0;
      for (long long e = 0; e < count; e++) {
        const double* el = elements + 9 * e;
        const double arg = mt * el[6] / t_fo;
        const double boost = std::exp((px * el[7] + py * el[8]) / t_fo);
        sum += (2 * mt * std::cyl_bessel_k(1.0, arg) * el[3] + 2 * std::cyl_bessel_k(0.0, arg) * (px * el[4] + py * el[5])) *
               boost;
      }
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
  if (!elements || count < 0 || !(t_fo > 0) || mass < 0 || !pt || !phi || npt < 1 || nphi < 1 || !out)
    return VH_E_ARG;
  const double pref = degeneracy / (8 * M_PI * M_PI * M_PI);
  for (int a = 0; a < npt; a++)
    for (int b = 0; b < nphi; b++) {
      const double mt = std::sqrt(mass * mass + pt[a] * pt[a]);
      const double px = pt[a] * std::cos(phi[b]), py = pt[a] * std::sin(phi[b]);
      double sum = 0;
      for (long long e = 0; e < count; e++) {
        const double* el = elements + 12 * e;
        const double tau = el[0], eta = el[3];
        const double pt_ = mt * std::cosh(y - eta), pe = mt * std::sinh(y - eta) / tau;
        const double pds = pt_ * el[4] + px * el[5] + py * el[6] + pe * el[7];
        const double pu = pt_ * el[8] - px * el[9] - py * el[10] - tau * tau * pe * el[11];
        sum += pds * std::exp(-pu / t_fo);
      }
      out[(long long)a * nphi + b] = pref * sum;
    }
  return VH_OK;
}
