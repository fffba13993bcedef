// Initialisation, reduction and diagnostic kernels around the step.
#pragma once

#include "vh_kernels.cuh"

namespace vh {

// T^{tau mu} = (e+P) u^tau u^mu - P g^{tau mu} + pi^{tau mu} on every cell
// of set A (NEWEST5/init.h:539-549, NEWEST5/Source.h:618-626).
template <class R>
__global__ void k_fill_tmunu(DevCfg C, DevPtrs<R> P, double tau) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C.n || c % C.px >= C.gx) return;  // padding cells stay untouched
  const R t2 = C.cart ? (R)1 : (R)(tau * tau);
  R u[4], p[5];
  const R e = P.e()[c];
#pragma unroll
  for (int l = 0; l < 4; l++) u[l] = P.u(l)[c];
#pragma unroll
  for (int l = 0; l < 5; l++) p[l] = P.A(4 + l)[c];
  const R Pp = eos_P<R>(C, e), ep = e + Pp;
  PiDep<R> d = pi_dep<R>(u[0], u[1], u[2], u[3], p, t2);
  P.A(0)[c] = -Pp + ep * (u[0] * u[0]) + d.tt;
  P.A(1)[c] = ep * u[0] * u[1] + d.tx;
  P.A(2)[c] = ep * u[0] * u[2] + d.ty;
  P.A(3)[c] = ep * u[0] * u[3] + d.te;
}

// Primitive fields of every cell into 17 x n doubles: e, P, T, u^mu (4) and
// the ten pi^{mu nu} (tt, tx, ty, te, xx, xy, xe, yy, ye, ee), the dependent
// components by transversality and tracelessness (the reference cell's En, P,
// Temp, u[4] and pi; NEWEST5/maindef.h:392-466, 497-501).
template <class R>
__global__ void k_primitive(DevCfg C, DevPtrs<R> P, double tau, double* out) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = C.n;
  if (c >= n || c % C.px >= C.gx) return;  // not the padding cells
  const R t2 = C.cart ? (R)1 : (R)(tau * tau);
  R u[4], p[5];
  const R e = P.e()[c];
#pragma unroll
  for (int l = 0; l < 4; l++) u[l] = P.u(l)[c];
#pragma unroll
  for (int l = 0; l < 5; l++) p[l] = P.A(4 + l)[c];
  R Pp, cs2, T;
  eos_all<R>(C, e, Pp, cs2, T);
  const PiDep<R> d = pi_dep<R>(u[0], u[1], u[2], u[3], p, t2);
  out[c] = (double)e;
  out[n + c] = (double)Pp;
  out[2 * n + c] = (double)T;
#pragma unroll
  for (int l = 0; l < 4; l++) out[(3 + l) * n + c] = (double)u[l];
  const R pi10[10] = {d.tt, d.tx, d.ty, d.te, p[0], p[2], p[3], p[1], p[4], d.ee};
#pragma unroll
  for (int l = 0; l < 10; l++) out[(7 + l) * n + c] = (double)pi10[l];
}

// Landau matching of one cell (NEWEST5/ginit.h:521-656): the timelike
// eigenvector u of T^mu_nu = T^{mu a} g_{a nu} and its eigenvalue e.  The
// reference takes all four eigenpairs from GSL and keeps the one real pair
// with |v| < 1; here Rayleigh-quotient iteration starts from the flow of
// energy u ~ T^{tau mu} (the timelike pair is the one it reaches for any
// tensor with e > |p_i|), with the 4x4 solves of the root-find.  Returns
// false when the iteration leaves the light cone or does not converge.
VH_HD inline bool landau_cell(const double* T10, double tau, bool cart, double& e, double* u) {
  const double t2 = cart ? 1.0 : tau * tau;
  const double g[4] = {1.0, -1.0, -1.0, -t2};
  const int I[4][4] = {{0, 1, 2, 3}, {1, 4, 5, 6}, {2, 5, 7, 8}, {3, 6, 8, 9}};
  double M[4][4];
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) M[a][b] = T10[I[a][b]] * g[b];
  auto lnorm = [&](const double* x) { return x[0] * x[0] - x[1] * x[1] - x[2] * x[2] - t2 * x[3] * x[3]; };
  auto rayleigh = [&](const double* x) {
    double s = 0;
    for (int a = 0; a < 4; a++) {
      double r = 0;
      for (int b = 0; b < 4; b++) r += M[a][b] * x[b];
      s += g[a] * x[a] * r;
    }
    return s;
  };
  double x[4] = {T10[0], T10[1], T10[2], T10[3]};
  double nn = lnorm(x);
  if (!(nn > 0) || !(x[0] > 0)) { x[0] = 1; x[1] = x[2] = x[3] = 0; nn = 1; }
  const double in = 1.0 / sqrt(nn);
  for (int a = 0; a < 4; a++) u[a] = x[a] * in;
  double sig = rayleigh(u);
  bool conv = false;
  for (int it = 0; it < 60 && !conv; it++) {
    double A[4][4], y[4] = {u[0], u[1], u[2], u[3]};
    for (int a = 0; a < 4; a++)
      for (int b = 0; b < 4; b++) A[a][b] = M[a][b] - (a == b ? sig : 0.0);
    if (!solve4(A, y)) { conv = true; break; }  // sig is an eigenvalue to working precision
    const double ny = lnorm(y);
    if (!(ny > 0)) return false;
    const double s = (y[0] > 0 ? 1.0 : -1.0) / sqrt(ny);
    double d = 0;
    for (int a = 0; a < 4; a++) {
      const double v = y[a] * s;
      d = fmax(d, fabs(v - u[a]));
      u[a] = v;
    }
    sig = rayleigh(u);
    // the iteration converges cubically; a change of a few ulps is rounding
    // noise, so 1e-14 (not 1e-15, where noise can keep it going) ends it
    if (d <= 1e-14 * fabs(u[0])) conv = true;
  }
  if (!conv) return false;
  // the pair must be an eigenpair: |M u - e u| small against e u^tau
  double res = 0;
  for (int a = 0; a < 4; a++) {
    double r = -sig * u[a];
    for (int b = 0; b < 4; b++) r += M[a][b] * u[b];
    res = fmax(res, fabs(r));
  }
  e = sig;
  // timelike and future-directed by construction (positive norm, u^tau > 0;
  // at rest u^tau can round to 1 - 1 ulp)
  return u[0] > 0 && e > 0 && res <= 1e-10 * fabs(e) * u[0];
}

template <class R>
__global__ void k_landau(long long n, double tau, int cart, const double* T10, double* e, double* u4,
                         unsigned long long* nfail) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  double t[10], ee = 0, u[4] = {1, 0, 0, 0};
#pragma unroll
  for (int l = 0; l < 10; l++) t[l] = T10[(long long)l * n + c];
  if (!landau_cell(t, tau, cart != 0, ee, u)) atomicAdd(nfail, 1ull);
  e[c] = ee;
#pragma unroll
  for (int l = 0; l < 4; l++) u4[(long long)l * n + c] = u[l];
}

// Initial state from T^{mu nu} on every cell: Landau matching, then
// pi^{mu nu} = T^{mu nu} - (e + P) u^mu u^nu + P g^{mu nu} (its five evolved
// components), prevu = u; T^{tau mu} follows from k_fill_tmunu.
template <class R>
__global__ void k_init_tmunu(DevCfg C, DevPtrs<R> P, double tau, const double* T10, unsigned long long* nfail) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = C.n;
  if (c >= n || c % C.px >= C.gx) return;  // not the padding cells
  double t[10], e = 0, u[4] = {1, 0, 0, 0};
#pragma unroll
  for (int l = 0; l < 10; l++) t[l] = T10[(long long)l * n + c];
  if (!landau_cell(t, tau, C.cart, e, u)) atomicAdd(nfail, 1ull);
  double Pp, cs2, Te;
  eos_all<double>(C, e, Pp, cs2, Te);
  const double t2 = C.cart ? 1.0 : tau * tau;
  // evolved components xx, yy, xy, x-eta, y-eta at T10 indices 4, 7, 5, 6, 8
  const int q[5] = {4, 7, 5, 6, 8}, a5[5] = {1, 2, 1, 1, 2}, b5[5] = {1, 2, 2, 3, 3};
  const double gi[4] = {1.0, -1.0, -1.0, -1.0 / t2};
  P.e()[c] = (R)e;
#pragma unroll
  for (int l = 0; l < 4; l++) { P.u(l)[c] = (R)u[l]; P.pu(l)[c] = (R)u[l]; }
  // NEWEST5/ginit.h:955-989: the ideal tensor tid, its trace e - 3P taken
  // off as PI (g - u u) with PI = -trace/3, so that pi is traceless; PI
  // itself is not evolved
  double tid[4];
#pragma unroll
  for (int a = 0; a < 4; a++) tid[a] = (e + Pp) * u[a] * u[a] - Pp * gi[a];
  const double PI = -(tid[0] - tid[1] - tid[2] - t2 * tid[3]) / 3.0;
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const int a = a5[k], b = b5[k];
    const double id = (e + Pp) * u[a] * u[b] - (a == b ? Pp * gi[a] : 0.0);
    const double pim = PI * ((a == b ? gi[a] : 0.0) - u[a] * u[b]);
    P.A(4 + k)[c] = (R)(t[q[k]] - id - pim);
  }
}

// prevu from T^{mu nu} one step before the initial time (the reference's
// ginit at tau - ts, NEWEST5/ginit.h:945-953): Landau matching, u only.
template <class R>
__global__ void k_prevu_tmunu(DevCfg C, DevPtrs<R> P, double tau, const double* T10, unsigned long long* nfail) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = C.n;
  if (c >= n || c % C.px >= C.gx) return;  // not the padding cells
  double t[10], e = 0, u[4] = {1, 0, 0, 0};
#pragma unroll
  for (int l = 0; l < 10; l++) t[l] = T10[(long long)l * n + c];
  if (!landau_cell(t, tau, C.cart, e, u)) atomicAdd(nfail, 1ull);
#pragma unroll
  for (int l = 0; l < 4; l++) P.pu(l)[c] = (R)u[l];
}

// Velocity gradients with the coverage the reference's CalcDer4Vel has
// (NEWEST5/Source.h:3-101): d_tau on the interior; d_x for i in [2, gx-3]
// on interior (j,k); d_y likewise; d_eta for every k on interior (i,j) with
// the edge stencils clamped; zero elsewhere.  Written to du16 (16 x n).
template <class R>
__global__ void k_du_full(DevCfg C, DevPtrs<R> P, R* du16, double ts) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C.n) return;
  const int i = (int)(c % C.px), j = (int)((c / C.px) % C.gy), k = (int)(c / ((long long)C.px * C.gy));
  const bool ii = i >= C.il && i < C.ir, jj = j >= C.jl && j < C.jr, kk = k >= C.kl && k < C.kr;
#pragma unroll 1
  for (int l = 0; l < 4; l++) {
    const R* u = P.u(l);
    R d0 = 0, d1 = 0, d2 = 0, d3 = 0;
    if (ii && jj && kk) d0 = (u[c] - P.pu(l)[c]) / (R)ts;
    if (jj && kk && i >= 2 && i < C.gx - 2) {
      const R L = weno_left<R>(u[c - 2], u[c - 1], u[c], u[c + 1], u[c + 2]);
      const R Rr = weno_right<R>(u[c - 2], u[c - 1], u[c], u[c + 1], u[c + 2]);
      d1 = (L - Rr) / (R)C.dx;
    }
    if (ii && kk && j >= 2 && j < C.gy - 2) {
      const long long s = C.px;
      const R L = weno_left<R>(u[c - 2 * s], u[c - s], u[c], u[c + s], u[c + 2 * s]);
      const R Rr = weno_right<R>(u[c - 2 * s], u[c - s], u[c], u[c + s], u[c + 2 * s]);
      d2 = (L - Rr) / (R)C.dy;
    }
    if (!C.bi && ii && jj) {
      const long long s = (long long)C.px * C.gy;
      const int Z = C.gz;
      R qm2, qm1, qc = u[c], qp1, qp2;
      if (k > 1 && k < Z - 2) { qm1 = u[c - s]; qm2 = u[c - 2 * s]; qp1 = u[c + s]; qp2 = u[c + 2 * s]; }
      else if (k == 0) { qm2 = qm1 = qc; qp1 = u[c + s]; qp2 = u[c + 2 * s]; }
      else if (k == 1) { qm2 = qm1 = u[c - s]; qp1 = u[c + s]; qp2 = u[c + 2 * s]; }
      else if (k == Z - 2) { qm1 = u[c - s]; qm2 = u[c - 2 * s]; qp2 = qp1 = u[c + s]; }
      else { qm1 = u[c - s]; qm2 = u[c - 2 * s]; qp2 = qp1 = qc; }
      const R L = weno_left<R>(qm2, qm1, qc, qp1, qp2);
      const R Rr = weno_right<R>(qm2, qm1, qc, qp1, qp2);
      d3 = (L - Rr) / (R)C.dz;
    }
    du16[(l * 4 + 0) * C.n + c] = d0;
    du16[(l * 4 + 1) * C.n + c] = d1;
    du16[(l * 4 + 2) * C.n + c] = d2;
    du16[(l * 4 + 3) * C.n + c] = d3;
  }
}

// Navier-Stokes pi = 2 eta sigma on every cell from du16
// (NEWEST5/Source.h:535-605, NSInit 607-630).
template <class R>
__global__ void k_ns_pi(DevCfg C, DevPtrs<R> P, const R* du16, double tau) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C.n || c % C.px >= C.gx) return;  // not the padding cells
  R u[4], du[4][4];
  const R e = P.e()[c];
#pragma unroll
  for (int l = 0; l < 4; l++) u[l] = P.u(l)[c];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) du[a][b] = du16[(a * 4 + b) * C.n + c];
  const R Pp = eos_P<R>(C, e);
  R eta, tp;
  transport<R>(C, e, Pp, &eta, &tp);
  R sig[4][4], th, acc[4];
  is_kinematics<R>(C.cart, (R)tau, u, du, sig, th, acc);
  P.A(4)[c] = (R)2 * eta * sig[1][1];
  P.A(5)[c] = (R)2 * eta * sig[2][2];
  P.A(6)[c] = (R)2 * eta * sig[1][2];
  P.A(7)[c] = (R)2 * eta * sig[1][3];
  P.A(8)[c] = (R)2 * eta * sig[2][3];
}

// Navier-Stokes shear 2 eta sigma^{mu nu}, all ten components (tt, tx, ty,
// t-eta, xx, xy, x-eta, yy, y-eta, eta-eta) on every cell from du16, in
// FP64 whatever the state's type: out10[q*n + c].  NEWEST10/Source.h:643-753
// (CalcNS) expands the same tensor into polynomials of u and du.
template <class R>
__global__ void k_ns_pi10(DevCfg C, DevPtrs<R> P, const R* du16, double tau, double* out10) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C.n || c % C.px >= C.gx) return;  // not the padding cells
  double u[4], du[4][4];
  const double e = (double)P.e()[c];
#pragma unroll
  for (int l = 0; l < 4; l++) u[l] = (double)P.u(l)[c];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) du[a][b] = (double)du16[(a * 4 + b) * C.n + c];
  double eta, tp;
  transport<double>(C, e, eos_P<double>(C, e), &eta, &tp);
  double sig[4][4], th, acc[4];
  is_kinematics<double, true>(C.cart, tau, u, du, sig, th, acc);
  const int MU[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3}, NU[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};
#pragma unroll
  for (int q = 0; q < 10; q++) out10[q * C.n + c] = 2.0 * eta * sig[MU[q]][NU[q]];
}

// Sources at the current state for the debug dump (interior only).
template <class R>
__global__ void k_debug_src(DevCfg C, DevPtrs<R> P, const R* du16, R* src9, double tau) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C.n) return;
  const int i = (int)(c % C.px), j = (int)((c / C.px) % C.gy), k = (int)(c / ((long long)C.px * C.gy));
  for (int l = 0; l < 9; l++) src9[l * C.n + c] = 0;
  if (!(i >= C.il && i < C.ir && j >= C.jl && j < C.jr && k >= C.kl && k < C.kr)) return;
  R u[4], p[5], du[4][4];
  const R e = P.e()[c];
#pragma unroll
  for (int l = 0; l < 4; l++) u[l] = P.u(l)[c];
#pragma unroll
  for (int l = 0; l < 5; l++) p[l] = P.A(4 + l)[c];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) du[a][b] = du16[(a * 4 + b) * C.n + c];
  const R ts = (R)tau;
  if (!C.cart) {
    const R t2 = ts * ts, Pp = eos_P<R>(C, e), ep = e + Pp;
    PiDep<R> d = pi_dep<R>(u[0], u[1], u[2], u[3], p, t2);
    src9[0 * C.n + c] = -Pp - t2 * (d.ee + ep * u[3] * u[3]);
    src9[3 * C.n + c] = -(R)2 * (d.te + ep * u[0] * u[3]);
  }
  R s5[5];
  is_source<R>(C, ts, e, u, p, du, s5);
  if (C.cart && !C.bi && (k - C.kl) >= C.nz - NG) s5[0] = s5[1] = s5[2] = s5[3] = s5[4] = 0;
  for (int q = 0; q < 5; q++) src9[(4 + q) * C.n + c] = s5[q];
}

// ---------------------------------------------------------- reductions

__device__ inline void atomic_max_nonneg(unsigned long long* slot, double v) {
  // the bit patterns of non-negative doubles order like the values
  atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}

// max over the interior of hbarc * T(e) (NEWEST5/utils.h:263-283)
template <class R>
__global__ void k_max_temp(DevCfg C, DevPtrs<R> P, unsigned long long* out) {
  const long long nint = (long long)C.nx * C.ny * (C.kr - C.kl);
  double m = 0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += (long long)gridDim.x * blockDim.x) {
    const int i = C.il + (int)(t % C.nx), j = C.jl + (int)((t / C.nx) % C.ny);
    const int k = C.kl + (int)(t / ((long long)C.nx * C.ny));
    const double T = C.hbarc * (double)eos_T<R>(C, P.e()[cix(C, i, j, k)]);
    m = fmax(m, T);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, m);
}

// Neumaier-compensated sums of tau T^{tau mu} dV over the interior of set A.
// One (sum, compensation) pair per block and component into part[4][2][nb].
__device__ inline void two_sum_add(double& s, double& c, double v) {
  const double t = s + v;
  if (fabs(s) >= fabs(v)) c += (s - t) + v; else c += (v - t) + s;
  s = t;
}
template <class R>
__global__ void k_conserve_part(DevCfg C, DevPtrs<R> P, double tau, double dv, double* part) {
  const long long nint = (long long)C.nx * C.ny * (C.kr - C.kl);
  double s[4] = {0, 0, 0, 0}, cc[4] = {0, 0, 0, 0};
  const double tf = C.cart ? 1.0 : tau;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += (long long)gridDim.x * blockDim.x) {
    const int i = C.il + (int)(t % C.nx), j = C.jl + (int)((t / C.nx) % C.ny);
    const int k = C.kl + (int)(t / ((long long)C.nx * C.ny));
    const long long c = cix(C, i, j, k);
#pragma unroll
    for (int l = 0; l < 4; l++) two_sum_add(s[l], cc[l], tf * (double)P.A(l)[c] * dv);
  }
  __shared__ double sh[2][4][256];
#pragma unroll
  for (int l = 0; l < 4; l++) { sh[0][l][threadIdx.x] = s[l]; sh[1][l][threadIdx.x] = cc[l]; }
  __syncthreads();
  if (threadIdx.x < 4) {
    const int l = threadIdx.x;
    double S = 0, Cc = 0;
    for (int q = 0; q < (int)blockDim.x; q++) { two_sum_add(S, Cc, sh[0][l][q]); Cc += sh[1][l][q]; }
    part[(l * 2 + 0) * gridDim.x + blockIdx.x] = S;
    part[(l * 2 + 1) * gridDim.x + blockIdx.x] = Cc;
  }
}
static __global__ void k_conserve_final(const double* part, int nb, double* out4) {
  const int l = threadIdx.x;
  if (l >= 4) return;
  double S = 0, Cc = 0;
  for (int q = 0; q < nb; q++) { two_sum_add(S, Cc, part[(l * 2) * nb + q]); Cc += part[(l * 2 + 1) * nb + q]; }
  out4[l] = S + Cc;
}

// Largest sqrt(ax^2 + ay^2 + az^2) of the face signal speeds right of each
// interior cell (NEWEST5/hydroKT.h:317-344 CFL).
template <class R>
__global__ void k_cfl(DevCfg C, DevPtrs<R> P, double tau, unsigned long long* out) {
  const long long nint = (long long)C.nx * C.ny * (C.kr - C.kl);
  double m = 0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += (long long)gridDim.x * blockDim.x) {
    const int i = C.il + (int)(t % C.nx), j = C.jl + (int)((t / C.nx) % C.ny);
    const int k = C.kl + (int)(t / ((long long)C.nx * C.ny));
    double a2 = 0;
    for (int d = 0; d < (C.bi ? 2 : 3); d++) {
      const long long s = d == 0 ? 1 : (d == 1 ? (long long)C.px : (long long)C.px * C.gy);
      const int pos = d == 0 ? i : (d == 1 ? j : k);
      const int lo = d == 0 ? C.il : (d == 1 ? C.jl : C.kl), hi = d == 0 ? C.ir : (d == 1 ? C.jr : C.kr);
      R q[6];
      for (int o = -2; o <= 3; o++) {
        const int g = pos + o;
        R v = 0;
        if (g >= lo && g < hi) {
          const long long cc = cix(C, i, j, k) + (long long)o * s;
          const R u0 = P.u(0)[cc];
          v = d == 0 ? P.u(1)[cc] / u0 : (d == 1 ? P.u(2)[cc] / u0 : (C.cart ? P.u(3)[cc] / u0 : (R)tau * P.u(3)[cc] / u0));
        }
        q[o + 2] = v;
      }
      const R sl = weno_left<R>(q[0], q[1], q[2], q[3], q[4]);
      const R sr = weno_right<R>(q[1], q[2], q[3], q[4], q[5]);
      const double a = fmax(fabs((double)sl), fabs((double)sr));
      a2 += a * a;
    }
    m = fmax(m, sqrt(a2));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, m);
}

// precision conversion between the canonical double layout and float state
static __global__ void k_d2f(const double* in, float* out, long long n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = (float)in[t];
}
static __global__ void k_f2d(const float* in, double* out, long long n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = (double)in[t];
}

}  // namespace vh
