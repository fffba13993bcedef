// Isothermal freeze-out hypersurface and Boltzmann Cooper-Frye spectra: the
// arithmetic of one space-time cube and of one (element, momentum) term,
// shared by the host entry points (vh_freezeout.cpp) and the device kernels
// (vh_freezeout_dev.cu), so that both emit the same elements in the same
// order.  The reference stops at the freeze-out temperature
// (NEWEST5/main.cpp:201-204, MaxTempGev in utils.h:263) and has no
// hypersurface; this is the step after the path.
//
// The surface T = T_fo is taken on the piecewise-linear interpolant of T
// between two time slices: each space-time cube between neighbouring cell
// centres is split into Kuhn simplices around its main diagonal (one per
// order of the axes: 6 tetrahedra in (tau, x, y), 24 4-simplices in
// (tau, x, y, eta)), and each simplex cut by the isotherm gives a triangle
// or quadrilateral (2+1D) or a tetrahedron or triangular prism (3+1D),
// emitted as triangles / tetrahedra with the covariant normal
// dSigma_mu = tau eps_{mu ...} e1 e2 (...) / n!, oriented from the hot side
// to the cold side, and u^mu interpolated at the centroid.
#pragma once
#include <math.h>

#include <cmath>

#ifdef __CUDACC__
#define VH_FO_HD __host__ __device__ inline
#else
#define VH_FO_HD inline
#endif

namespace vh_fo {

constexpr int kG = 3;       // ghost layers per face
constexpr int kW2 = 9;      // doubles per 2+1D element: centroid(3), dSigma(3), u(3)
constexpr int kW3 = 12;     // doubles per 3+1D element: centroid(4), dSigma(4), u(4)
constexpr int kMax2 = 12;   // elements per cube at most: 6 tetrahedra x 2 triangles
constexpr int kMax3 = 72;   // 24 4-simplices x 3 tetrahedra

// the grid of one freeze-out call; D = 3 (tau, x, y) or 4 (tau, x, y, eta)
struct Geo {
  int nx, ny, nz;     // interior cells (nz = 1 for 2+1D)
  int gx, gy;         // ghost-inclusive extents in x, y
  long long n;        // ghost-inclusive cells of one slice
  double dx, dy, dz;  // cell sizes
  double x0, y0, z0;  // coordinate of the first interior cell
  double tau0, tau1, t_fo;
};

inline Geo make_geo(int nx, int ny, int nz, double dx, double dy, double dz, double tau0, double tau1, double t_fo,
                    bool bi) {
  Geo g;
  g.nx = nx; g.ny = ny; g.nz = bi ? 1 : nz;
  g.gx = nx + 2 * kG; g.gy = ny + 2 * kG;
  g.n = (long long)g.gx * g.gy * (bi ? 1 : nz + 2 * kG);
  g.dx = dx; g.dy = dy; g.dz = dz;
  g.x0 = -((double)(nx / 2) * dx); g.y0 = -((double)(ny / 2) * dy); g.z0 = bi ? 0.0 : -((double)(nz / 2) * dz);
  g.tau0 = tau0; g.tau1 = tau1; g.t_fo = t_fo;
  return g;
}

// cubes of one call: (nx - 1)(ny - 1) in 2+1D, times (nz - 1) in 3+1D, x
// fastest, and the ghost-inclusive indices of cube c's lowest corner
VH_FO_HD long long cubes(const Geo& g, int D) {
  return (long long)(g.nx - 1) * (g.ny - 1) * (D == 4 ? g.nz - 1 : 1);
}
VH_FO_HD void cube_ijk(const Geo& g, long long c, int* i, int* j, int* k) {
  *i = (int)(c % (g.nx - 1)) + kG;
  c /= (g.nx - 1);
  *j = (int)(c % (g.ny - 1)) + kG;
  *k = (int)(c / (g.ny - 1)) + kG;
}

// vertex bits of Kuhn simplex s (0 <= s < m!) of the unit m-cube: the
// path 0 -> e_a -> e_a + e_b -> ... -> 2^m - 1 along the s-th permutation
// of the axes in lexicographic order (factorial-base digits of s)
VH_FO_HD void kuhn_simplex(int s, int m, int* v) {
  int avail[4] = {0, 1, 2, 3}, f = 1, bits = 0;
  for (int q = 2; q < m; q++) f *= q;  // (m - 1)!
  v[0] = 0;
  for (int q = 0; q < m; q++) {
    const int left = m - 1 - q;  // axes still to place after this one
    const int d = s / f;
    s %= f;
    const int axis = avail[d];
    for (int r = d; r < left; r++) avail[r] = avail[r + 1];
    bits |= 1 << axis;
    v[q + 1] = bits;
    if (left > 0) f /= left;
  }
}

// corner v of a cube: bit q set for the upper end of axis q (0 tau, 1 x,
// 2 y, 3 eta); lo, hi: the two coordinates per axis; f = T - T_fo
template <int D>
struct Corners {
  double lo[D], hi[D], u[1 << D][D], f[1 << D];
  VH_FO_HD double x(int v, int q) const { return ((v >> q) & 1) ? hi[q] : lo[q]; }
};

// cell index of corner v of cube (i, j, k) in its time slice
template <int D>
VH_FO_HD long long corner_cell(const Geo& g, int i, int j, int k, int v) {
  const int bx = (v >> 1) & 1, by = (v >> 2) & 1, bz = D == 4 ? (v >> 3) & 1 : 0;
  return ((long long)(k + bz - (D == 4 ? 0 : kG)) * g.gy + (j + by)) * g.gx + (i + bx);
}

// loads the corners of cube (i, j, k); returns false, having read T alone,
// when the isotherm misses it (all corners on one side)
template <int D>
VH_FO_HD bool load(const Geo& g, int i, int j, int k, const double* t0, const double* t1, const double* u0,
                   const double* u1, Corners<D>& K) {
  bool pos = false, neg = false;
  for (int v = 0; v < (1 << D); v++) {
    K.f[v] = ((v & 1) ? t1 : t0)[corner_cell<D>(g, i, j, k, v)] - g.t_fo;
    if (K.f[v] > 0) pos = true; else neg = true;
  }
  if (!pos || !neg) return false;
  K.lo[0] = g.tau0;
  K.hi[0] = g.tau1;
  K.lo[1] = g.x0 + (i - kG) * g.dx;
  K.hi[1] = g.x0 + (i + 1 - kG) * g.dx;
  K.lo[2] = g.y0 + (j - kG) * g.dy;
  K.hi[2] = g.y0 + (j + 1 - kG) * g.dy;
  if (D == 4) {
    K.lo[D - 1] = g.z0 + (k - kG) * g.dz;
    K.hi[D - 1] = g.z0 + (k + 1 - kG) * g.dz;
  }
  for (int v = 0; v < (1 << D); v++) {
    const long long c = corner_cell<D>(g, i, j, k, v);
    const double* U = (v & 1) ? u1 : u0;
    for (int q = 0; q < D; q++) K.u[v][q] = U[q * g.n + c];
  }
  return true;
}

// elements that cube (i, j, k) emits, from the signs of T - T_fo alone: per
// simplex cut by the isotherm, 1 (one vertex apart) or 2 triangles (two
// against two) in 2+1D, 1 or 3 tetrahedra (two against three) in 3+1D
template <int D>
VH_FO_HD int count(const Geo& g, int i, int j, int k, const double* t0, const double* t1) {
  unsigned hot = 0;
  for (int v = 0; v < (1 << D); v++)
    if (((v & 1) ? t1 : t0)[corner_cell<D>(g, i, j, k, v)] - g.t_fo > 0) hot |= 1u << v;
  if (hot == 0 || hot == (1u << (1 << D)) - 1) return 0;
  int total = 0, nsim = D == 4 ? 24 : 6;
  for (int s = 0; s < nsim; s++) {
    int v[5], nh = 0;
    kuhn_simplex(s, D, v);
    for (int q = 0; q <= D; q++) nh += (hot >> v[q]) & 1;
    const int nc = D + 1 - nh;
    if (!nh || !nc) continue;
    total += (nh == 1 || nc == 1) ? 1 : (D == 4 ? 3 : 2);
  }
  return total;
}

// the isotherm's crossing of edge a-b: position and u^mu
template <int D>
struct Pt {
  double x[D], u[D];
};
template <int D>
VH_FO_HD Pt<D> edge_point(const Corners<D>& K, int a, int b) {
  const double w = K.f[a] / (K.f[a] - K.f[b]);
  Pt<D> p;
  for (int q = 0; q < D; q++) {
    const double xa = K.x(a, q), xb = K.x(b, q);
    p.x[q] = xa + w * (xb - xa);
    p.u[q] = K.u[a][q] + w * (K.u[b][q] - K.u[a][q]);
  }
  return p;
}

// Element writer: element number `at` onwards into out (width doubles
// each), writing only below cap and counting every element.  On the host
// `at` starts at 0 and runs over the whole grid; on the device each cube
// starts at its offset in the exclusive scan of the per-cube counts.
struct Sink {
  double* out;
  long long at, cap;
  VH_FO_HD void put(const double* o, int width) {
    if (at < cap)
      for (int q = 0; q < width; q++) out[at * width + q] = o[q];
    at++;
  }
};

// triangle (a, b, c) of the 2+1D surface: dSigma_mu = (tau / 2)
// eps_{mu nu lambda} (b - a)^nu (c - a)^lambda per unit rapidity, oriented
// along cold - hot
VH_FO_HD void triangle(const Pt<3>& a, const Pt<3>& b, const Pt<3>& c, const double* cold, const double* hot, Sink& s) {
  double e1[3], e2[3], n[3], o[kW2];
  for (int q = 0; q < 3; q++) { e1[q] = b.x[q] - a.x[q]; e2[q] = c.x[q] - a.x[q]; }
  n[0] = 0.5 * (e1[1] * e2[2] - e1[2] * e2[1]);
  n[1] = 0.5 * (e1[2] * e2[0] - e1[0] * e2[2]);
  n[2] = 0.5 * (e1[0] * e2[1] - e1[1] * e2[0]);
  double d = 0;
  for (int q = 0; q < 3; q++) d += n[q] * (cold[q] - hot[q]);
  const double sg = d < 0 ? -1.0 : 1.0;
  const double tc = (a.x[0] + b.x[0] + c.x[0]) / 3;
  for (int q = 0; q < 3; q++) o[q] = (a.x[q] + b.x[q] + c.x[q]) / 3;
  for (int q = 0; q < 3; q++) o[3 + q] = sg * tc * n[q];
  for (int q = 0; q < 3; q++) o[6 + q] = (a.u[q] + b.u[q] + c.u[q]) / 3;
  s.put(o, kW2);
}

// tetrahedron (a, b, c, d) of the 3+1D surface: dSigma_mu = (tau / 6)
// eps_{mu nu lambda rho} e1^nu e2^lambda e3^rho, the cofactors of the
// matrix [unit_mu; e1; e2; e3], oriented along cold - hot
VH_FO_HD void tetra(const Pt<4>& a, const Pt<4>& b, const Pt<4>& c, const Pt<4>& d, const double* cold,
                    const double* hot, Sink& s) {
  double e[3][4], n[4], o[kW3];
  for (int q = 0; q < 4; q++) { e[0][q] = b.x[q] - a.x[q]; e[1][q] = c.x[q] - a.x[q]; e[2][q] = d.x[q] - a.x[q]; }
  for (int m = 0; m < 4; m++) {
    int cols[3], k = 0;
    for (int q = 0; q < 4; q++)
      if (q != m) cols[k++] = q;
    const double det = e[0][cols[0]] * (e[1][cols[1]] * e[2][cols[2]] - e[1][cols[2]] * e[2][cols[1]]) -
                       e[0][cols[1]] * (e[1][cols[0]] * e[2][cols[2]] - e[1][cols[2]] * e[2][cols[0]]) +
                       e[0][cols[2]] * (e[1][cols[0]] * e[2][cols[1]] - e[1][cols[1]] * e[2][cols[0]]);
    n[m] = ((m & 1) ? -det : det) / 6.0;
  }
  double dd = 0;
  for (int q = 0; q < 4; q++) dd += n[q] * (cold[q] - hot[q]);
  const double sg = dd < 0 ? -1.0 : 1.0;
  const double tc = (a.x[0] + b.x[0] + c.x[0] + d.x[0]) / 4;
  for (int q = 0; q < 4; q++) o[q] = (a.x[q] + b.x[q] + c.x[q] + d.x[q]) / 4;
  for (int q = 0; q < 4; q++) o[4 + q] = sg * tc * n[q];
  for (int q = 0; q < 4; q++) o[8 + q] = (a.u[q] + b.u[q] + c.u[q] + d.u[q]) / 4;
  s.put(o, kW3);
}

// every element of cube (i, j, k) in 2+1D (k unused): marching tetrahedra
VH_FO_HD void cube2(const Geo& g, int i, int j, const double* t0, const double* t1, const double* u0,
                    const double* u1, Sink& s) {
  Corners<3> K;
  if (!load<3>(g, i, j, kG, t0, t1, u0, u1, K)) return;
  for (int sx = 0; sx < 6; sx++) {
    int v[4], hot[4], cold[4], nh = 0, nc = 0;
    kuhn_simplex(sx, 3, v);
    for (int q = 0; q < 4; q++) {
      if (K.f[v[q]] > 0) hot[nh++] = v[q]; else cold[nc++] = v[q];
    }
    if (!nh || !nc) continue;
    double ph[3], pc[3];  // a hot and a cold corner: the orientation
    for (int q = 0; q < 3; q++) {
      ph[q] = K.x(hot[0], q);
      pc[q] = K.x(cold[0], q);
    }
    if (nh == 1 || nc == 1) {
      const int lone = nh == 1 ? hot[0] : cold[0];
      const int* o = nh == 1 ? cold : hot;
      triangle(edge_point(K, lone, o[0]), edge_point(K, lone, o[1]), edge_point(K, lone, o[2]), pc, ph, s);
    } else {
      // two against two: the quadrilateral a-b-c-d as two triangles
      const Pt<3> a = edge_point(K, hot[0], cold[0]), b = edge_point(K, hot[0], cold[1]);
      const Pt<3> c = edge_point(K, hot[1], cold[1]), d = edge_point(K, hot[1], cold[0]);
      triangle(a, b, c, pc, ph, s);
      triangle(a, c, d, pc, ph, s);
    }
  }
}

// every element of hypercube (i, j, k) in 3+1D: marching 4-simplices
VH_FO_HD void cube3(const Geo& g, int i, int j, int k, const double* t0, const double* t1, const double* u0,
                    const double* u1, Sink& s) {
  Corners<4> K;
  if (!load<4>(g, i, j, k, t0, t1, u0, u1, K)) return;
  for (int sx = 0; sx < 24; sx++) {
    int v[5], hot[5], cold[5], nh = 0, nc = 0;
    kuhn_simplex(sx, 4, v);
    for (int q = 0; q < 5; q++) {
      if (K.f[v[q]] > 0) hot[nh++] = v[q]; else cold[nc++] = v[q];
    }
    if (!nh || !nc) continue;
    double ph[4], pc[4];  // a hot and a cold corner: the orientation
    for (int q = 0; q < 4; q++) {
      ph[q] = K.x(hot[0], q);
      pc[q] = K.x(cold[0], q);
    }
    if (nh == 1 || nc == 1) {
      // one vertex against four: a tetrahedron
      const int lone = nh == 1 ? hot[0] : cold[0];
      const int* o = nh == 1 ? cold : hot;
      tetra(edge_point(K, lone, o[0]), edge_point(K, lone, o[1]), edge_point(K, lone, o[2]),
            edge_point(K, lone, o[3]), pc, ph, s);
    } else {
      // two against three: a triangular prism, as three tetrahedra
      const int* two = nh == 2 ? hot : cold;
      const int* three = nh == 2 ? cold : hot;
      const Pt<4> a0 = edge_point(K, two[0], three[0]), a1 = edge_point(K, two[0], three[1]);
      const Pt<4> a2 = edge_point(K, two[0], three[2]), b0 = edge_point(K, two[1], three[0]);
      const Pt<4> b1 = edge_point(K, two[1], three[1]), b2 = edge_point(K, two[1], three[2]);
      tetra(a0, a1, a2, b0, pc, ph, s);
      tetra(a1, a2, b0, b1, pc, ph, s);
      tetra(a2, b0, b1, b2, pc, ph, s);
    }
  }
}

// ------------------------------------------------------- Cooper-Frye terms
// momentum bins: p_T >= 0 and finite azimuths; for a massless hadron at
// p_T = 0 (m_T = 0) the boost-invariant term is a limit (m_T K1(m_T u/T) ->
// T/u) that its sum does not take, so there m_T = 0 is refused (host code)
inline bool bins_ok(double mass, const double* pt, int npt, const double* phi, int nphi, bool mt_zero_ok) {
  for (int a = 0; a < npt; a++)
    if (!(pt[a] >= 0) || !std::isfinite(pt[a]) || (pt[a] == 0 && mass == 0 && !mt_zero_ok)) return false;
  for (int b = 0; b < nphi; b++)
    if (!std::isfinite(phi[b])) return false;
  return true;
}

// Exponentially scaled modified Bessel functions e^z K0(z), e^z K1(z), z > 0,
// by the trapezoidal rule on K_nu(z) = int_0^inf exp(-z cosh t) cosh(nu t) dt
// (DLMF 10.32.9), whose error falls exponentially with 1/h for an integrand
// analytic in a strip (Trefethen and Weideman, SIAM Review 56 (2014) 385):
// e^z K_nu(z) = int exp(-2 z sinh^2(t/2)) cosh(nu t) dt with step
// h = min(1/4, 1/(2 sqrt z)), summed while 2 z sinh^2(t/2) <= 45.  Relative
// error within 4e-15 of the exact values for 1e-6 <= z <= 1e3 (74 nodes at
// most there; fewer as z grows).
VH_FO_HD void bessel_k01e(double z, double* k0e, double* k1e) {
  const double h = fmin(0.25, 0.5 / sqrt(z));
  double s0 = 0.5, s1 = 0.5;
  for (int q = 1; q < 4096; q++) {
    const double t = q * h, sh = sinh(0.5 * t), a = 2 * z * sh * sh;
    if (a > 45.0) break;
    const double g = exp(-a);
    s0 += g;
    s1 += g * cosh(t);
  }
  *k0e = h * s0;
  *k1e = h * s1;
}

// one element's term of the boost-invariant spectrum at (m_T, p_x, p_y):
// 2 m_T K1(a) dSigma_tau + 2 K0(a) (p_x dSigma_x + p_y dSigma_y) times
// exp((p_x u^x + p_y u^y) / T), a = m_T u^tau / T
VH_FO_HD double cf2_term(const double* el, double mt, double px, double py, double t_fo) {
  const double a = mt * el[6] / t_fo;
  double k0e, k1e;
  bessel_k01e(a, &k0e, &k1e);
  const double boost = exp((px * el[7] + py * el[8]) / t_fo - a);
  return (2 * mt * k1e * el[3] + 2 * k0e * (px * el[4] + py * el[5])) * boost;
}

// one element's term at rapidity y of the 3+1D spectrum: p^mu dSigma_mu
// exp(-p.u / T), p^tau = m_T cosh(y - eta), p^eta = m_T sinh(y - eta) / tau
VH_FO_HD double cf3_term(const double* el, double mt, double px, double py, double y, double t_fo) {
  const double tau = el[0], eta = el[3];
  const double pt_ = mt * cosh(y - eta), pe = mt * sinh(y - eta) / tau;
  const double pds = pt_ * el[4] + px * el[5] + py * el[6] + pe * el[7];
  const double pu = pt_ * el[8] - px * el[9] - py * el[10] - tau * tau * pe * el[11];
  return pds * exp(-pu / t_fo);
}

}  // namespace vh_fo
