// Device-side arithmetic of the viscous KT step, templated on the storage
// and flux precision R (double for the FP64 step, float for the mixed step).
// The conserved-to-primitive Newton solve and the EOS evaluations it makes
// are always double.  Each routine cites the reference lines it implements.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// host+device math: the same arithmetic also compiles for host-side checks
#define VH_HD __host__ __device__

namespace vh {

constexpr int NG = 3;  // ghost layers (NEWEST5/maindef.h:369-371 BORDER)

// Problem description passed by value to every kernel.
struct DevCfg {
  int gx, gy, gz;              // ghost-inclusive extents
  int px;                      // row pitch in cells (>= gx): a handle's rows are padded to 8 cells
  int xt0;                     // x of the first line of the y and eta sweeps' tiles (0 or il)
  int il, ir, jl, jr, kl, kr;  // interior bounds
  int nx, ny, nz;
  long long n;                 // px*gy*gz: cells per array, padding included
  int cart, bi, recon, mirror;
  double dx, dy, dz;
  int eos_kind;
  double eos_a;
  int eos_n;
  double eos_l0, eos_idl;       // log(e_0), 1/dlog(e)
  const double* eos_d;          // [4][eos_n] e, P, cs2, T (double)
  const float* eos_f;           // the same in float
  double etas0, etas1, etas_tc, hbarc;
  int taupi_kind;
  double taupi_c;               // tau_pi of VH_TAUPI_CONST
  int cold;                     // cold-plasma test: no -pi/tau_pi relaxation
  double mm_theta;
};

// Device buffers of one event: 52 ghost-inclusive SoA arrays of `stride`
// cells each.  Fields 0..17 are the canonical state (at base0), fields
// 18..51 the step's scratch (at base1); an event inside a batch pool is the
// same view shifted by its cell offset.
//   0 e, 1..4 u^mu, 5..9 pi (set A), 10..13 T^{tau mu} (set A), 14..17 prevu,
//   18..26 set B (T^{tau mu} 4, pi 5), 27..30 stage-1 tau T^{tau mu},
//   31..39 flux-divergence accumulator, 40..51 spatial du[l][1+d] at l*3+d.
template <class R>
struct DevPtrs {
  R* base0;
  R* base1;
  long long stride;
  unsigned int* status;            // OR of failure bits
  unsigned long long* iters;       // Newton iterations
  __host__ __device__ R* f(int q) const { return q < 18 ? base0 + (long long)q * stride : base1 + (long long)(q - 18) * stride; }
  __host__ __device__ R* e() const { return base0; }
  __host__ __device__ R* u(int l) const { return base0 + (long long)(1 + l) * stride; }
  __host__ __device__ R* pu(int l) const { return base0 + (long long)(14 + l) * stride; }
  // conserved set: A (step start) or B (stage 1); l < 4 T^{tau mu}, else pi
  __host__ __device__ R* A(int l) const { return base0 + (long long)(l < 4 ? 10 + l : l + 1) * stride; }
  __host__ __device__ R* B(int l) const { return base1 + (long long)l * stride; }
  __host__ __device__ R* S(int use_b, int l) const { return use_b ? B(l) : A(l); }
  __host__ __device__ R* v1t(int l) const { return base1 + (long long)(9 + l) * stride; }
  __host__ __device__ R* res(int l) const { return base1 + (long long)(13 + l) * stride; }
  __host__ __device__ R* du(int l) const { return base1 + (long long)(22 + l) * stride; }
  __host__ __device__ DevPtrs shifted(long long off) const {
    DevPtrs p = *this;
    p.base0 += off;
    p.base1 += off;
    return p;
  }
};

enum : unsigned { ST_ROOT = 1u, ST_CAUSAL = 2u, ST_NEGE = 4u, ST_TMA = 8u };

__host__ VH_HD inline long long cix(const DevCfg& C, int i, int j, int k) {
  return ((long long)k * C.gy + j) * C.px + i;
}

// ------------------------------------------------------------------ EOS

template <class R>
VH_HD inline const R* eos_tab(const DevCfg& C);
template <>
VH_HD inline const double* eos_tab<double>(const DevCfg& C) { return C.eos_d; }
template <>
VH_HD inline const float* eos_tab<float>(const DevCfg& C) { return C.eos_f; }

VH_HD inline double d_log(double x) { return log(x); }
VH_HD inline float d_log(float x) {
#ifdef __CUDA_ARCH__
  return __logf(x);
#else
  return logf(x);
#endif
}
VH_HD inline double d_sqrt(double x) { return sqrt(x); }
VH_HD inline float d_sqrt(float x) { return sqrtf(x); }

// Row i with e_i <= e < e_{i+1}: a log-based guess corrected against the
// nodes, so the bracket is exact whatever the rounding of log.
template <class R>
VH_HD inline int eos_row(const DevCfg& C, const R* t, R e) {
  const int n = C.eos_n;
  // a single-precision log is enough for the guess: the loops below make
  // the bracket exact
  int i = (int)((d_log((float)e) - (float)C.eos_l0) * (float)C.eos_idl);
  i = i < 0 ? 0 : (i > n - 2 ? n - 2 : i);
  while (i > 0 && e < t[i]) i--;
  while (i < n - 2 && e >= t[i + 1]) i++;
  return i;
}

// Synthetic tabulated EOS: linear in e between log-spaced rows; below the
// first row P = cs2_0 e and T ~ e^(1/4); above the last row P grows with the
// last cs2 and T ~ e^(1/4).
template <class R>
VH_HD inline void eos_table(const DevCfg& C, R e, R* P, R* cs2, R* T) {
  const R* t = eos_tab<R>(C);
  const int n = C.eos_n;
  const R* te = t;
  const R* tp = t + n;
  const R* tc = t + 2 * n;
  const R* tt = t + 3 * n;
  if (e <= te[0]) {
    *cs2 = tc[0];
    *P = tc[0] * e;
    *T = tt[0] * d_sqrt(d_sqrt(e / te[0]));
    return;
  }
  if (e >= te[n - 1]) {
    *cs2 = tc[n - 1];
    *P = tp[n - 1] + tc[n - 1] * (e - te[n - 1]);
    *T = tt[n - 1] * d_sqrt(d_sqrt(e / te[n - 1]));
    return;
  }
  int i = eos_row<R>(C, te, e);
  R w = (e - te[i]) / (te[i + 1] - te[i]);
  *P = tp[i] + w * (tp[i + 1] - tp[i]);
  *cs2 = tc[i] + w * (tc[i + 1] - tc[i]);
  *T = tt[i] + w * (tt[i + 1] - tt[i]);
}

// P(e) (NEWEST5/maindef.h:332 EOS)
template <class R>
VH_HD inline R eos_P(const DevCfg& C, R e) {
  if (C.eos_kind == 0) return e / (R)3;
  R P, c, T;
  eos_table<R>(C, e, &P, &c, &T);
  return P;
}
// dP/de (NEWEST5/maindef.h:333 DPDE)
template <class R>
VH_HD inline R eos_cs2(const DevCfg& C, R e) {
  if (C.eos_kind == 0) return (R)1 / (R)3;
  R P, c, T;
  eos_table<R>(C, e, &P, &c, &T);
  return c;
}
VH_HD inline double conf_T(double x) { return pow(x, 0.25); }
VH_HD inline float conf_T(float x) { return sqrtf(sqrtf(x)); }
// T(e) (NEWEST5/maindef.h:335 FT)
template <class R>
VH_HD inline R eos_T(const DevCfg& C, R e) {
  if (C.eos_kind == 0) return conf_T(e / (R)C.eos_a);
  R P, c, T;
  eos_table<R>(C, e, &P, &c, &T);
  return T;
}
// P, c_s^2 and T of one state (one table lookup)
template <class R>
VH_HD inline void eos_all(const DevCfg& C, R e, R& P, R& cs2, R& T) {
  if (C.eos_kind == 0) {
    P = e / (R)3;
    cs2 = (R)1 / (R)3;
    T = conf_T(e / (R)C.eos_a);
    return;
  }
  eos_table<R>(C, e, &P, &cs2, &T);
}
// eta = (eta/s)(T) s with s = (e+P)/T, and tau_pi (NEWEST5/maindef.h:336-339),
// from a known temperature
template <class R>
VH_HD inline void transport_T(const DevCfg& C, R e, R P, R T, R* eta, R* taupi) {
  R s = (e + P) / T;
  R tg = T * (R)C.hbarc - (R)C.etas_tc;
  R etas = (R)C.etas0 + (R)C.etas1 * (tg > (R)0 ? tg : (R)0);
  *eta = etas * s;
  *taupi = (C.taupi_kind == 1) ? (R)5 * (*eta) / (e + P) : C.taupi_kind == 2 ? (R)C.taupi_c : (R)1.5 * ((*eta) / P);
}
template <class R>
VH_HD inline void transport(const DevCfg& C, R e, R P, R* eta, R* taupi) {
  R T = eos_T<R>(C, e);
  R s = (e + P) / T;
  R tg = T * (R)C.hbarc - (R)C.etas_tc;
  R etas = (R)C.etas0 + (R)C.etas1 * (tg > (R)0 ? tg : (R)0);
  *eta = etas * s;
  *taupi = (C.taupi_kind == 1) ? (R)5 * (*eta) / (e + P) : C.taupi_kind == 2 ? (R)C.taupi_c : (R)1.5 * ((*eta) / P);
}

// --------------------------------------------------- pi closure (A1..A5)
// pi^{tau tau}, pi^{tau x}, pi^{tau y}, pi^{tau eta}, pi^{eta eta} from the
// evolved five by transversality and tracelessness in diag(1,-1,-1,-t2)
// (NEWEST5/maindef.h:497-501).
template <class R>
struct PiDep {
  R tt, tx, ty, te, ee;
};
template <class R>
VH_HD inline PiDep<R> pi_dep(R u0, R u1, R u2, R u3, const R* p, R t2) {
  PiDep<R> d;
  const R iD = (R)1 / (u0 * u0 - t2 * u3 * u3);
  const R iu0 = (R)1 / u0;
  const R Q = u1 * u1 * p[0] + (R)2 * u1 * u2 * p[2] + u2 * u2 * p[1] + (R)2 * t2 * u3 * (u1 * p[3] + u2 * p[4]);
  d.tt = (Q - t2 * u3 * u3 * (p[0] + p[1])) * iD;
  d.ee = (Q - u0 * u0 * (p[0] + p[1])) * iD / t2;
  d.tx = (p[0] * u1 + p[2] * u2 + p[3] * u3 * t2) * iu0;
  d.ty = (p[2] * u1 + p[1] * u2 + p[4] * u3 * t2) * iu0;
  d.te = (u1 * p[3] + u2 * p[4] + t2 * u3 * d.ee) * iu0;
  return d;
}

// ------------------------------------------------------------------ WENO5
// Jiang-Shu WENO5 with p = 2, eps = 1e-6 and linear weights (0.3,0.6,0.1)
// (NEWEST5/utils.h:57-160).  Evaluation order follows the reference.
template <class R>
VH_HD inline void weno_beta(R qm2, R qm1, R qc, R qp1, R qp2, R& b0, R& b1, R& b2) {
  const R c13 = (R)(13. / 12.);
  R a = qc - (R)2 * qp1 + qp2, c = (R)3 * qc - (R)4 * qp1 + qp2;
  b0 = c13 * (a * a) + (R)0.25 * (c * c);
  a = qm1 - (R)2 * qc + qp1; c = qm1 - qp1;
  b1 = c13 * (a * a) + (R)0.25 * (c * c);
  a = qm2 - (R)2 * qm1 + qc; c = qm2 - (R)4 * qm1 + (R)3 * qc;
  b2 = c13 * (a * a) + (R)0.25 * (c * c);
}
// The nonlinear weights w_k = a_k / sum(a), a_k = d_k / (eps + b_k)^2, are
// formed with a single division: multiplying every a_k by the product of
// the three (eps + b)^2 gives n_k = d_k prod_{j != k} (eps + b_j)^2, so the
// face value is sum(n_k q_k) / sum(n_k).  The 1/6 of the candidate
// polynomials is folded into the same division.  This is the reference's
// WENO5 (NEWEST5/utils.h:102-160) up to rounding.
// value at face i+1/2 from the stencil centred on i (genWENOL)
template <class R>
VH_HD inline R weno_left(R qm2, R qm1, R qc, R qp1, R qp2) {
  R b0, b1, b2;
  weno_beta<R>(qm2, qm1, qc, qp1, qp2, b0, b1, b2);
  const R eps = (R)1e-6;
  const R e0 = eps + b0, e1 = eps + b1, e2 = eps + b2;
  const R E0 = e0 * e0, E1 = e1 * e1, E2 = e2 * e2;
  const R n0 = (R)0.3 * (E1 * E2), n1 = (R)0.6 * (E0 * E2), n2 = (R)0.1 * (E0 * E1);
  const R q0 = (R)2 * qc + (R)5 * qp1 - qp2;
  const R q1 = -qm1 + (R)5 * qc + (R)2 * qp1;
  const R q2 = (R)2 * qm2 - (R)7 * qm1 + (R)11 * qc;
  return (n0 * q0 + n1 * q1 + n2 * q2) / ((R)6 * (n0 + n1 + n2));
}
// value at face i-1/2 from the stencil centred on i (genWENOR)
template <class R>
VH_HD inline R weno_right(R qm2, R qm1, R qc, R qp1, R qp2) {
  R b0, b1, b2;
  weno_beta<R>(qm2, qm1, qc, qp1, qp2, b0, b1, b2);
  const R eps = (R)1e-6;
  const R e0 = eps + b0, e1 = eps + b1, e2 = eps + b2;
  const R E0 = e0 * e0, E1 = e1 * e1, E2 = e2 * e2;
  const R n0 = (R)0.1 * (E1 * E2), n1 = (R)0.6 * (E0 * E2), n2 = (R)0.3 * (E0 * E1);
  const R q0 = (R)11 * qc - (R)7 * qp1 + (R)2 * qp2;
  const R q1 = (R)2 * qm1 + (R)5 * qc - qp1;
  const R q2 = -qm2 + (R)5 * qm1 + (R)2 * qc;
  return (n0 * q0 + n1 * q1 + n2 * q2) / ((R)6 * (n0 + n1 + n2));
}
// Both face values of one stencil at once: L at i+1/2 (genWENOL) and R at
// i-1/2 (genWENOR) share the smoothness indicators and their products.
template <class R>
VH_HD inline void weno_lr(R qm2, R qm1, R qc, R qp1, R qp2, R& L, R& Rr) {
  R b0, b1, b2;
  weno_beta<R>(qm2, qm1, qc, qp1, qp2, b0, b1, b2);
  const R eps = (R)1e-6;
  const R e0 = eps + b0, e1 = eps + b1, e2 = eps + b2;
  const R E0 = e0 * e0, E1 = e1 * e1, E2 = e2 * e2;
  const R P12 = E1 * E2, P02 = E0 * E2, P01 = E0 * E1;
  const R nl0 = (R)0.3 * P12, nl1 = (R)0.6 * P02, nl2 = (R)0.1 * P01;
  const R nr0 = (R)0.1 * P12, nr1 = nl1, nr2 = (R)0.3 * P01;
  const R ql0 = (R)2 * qc + (R)5 * qp1 - qp2;
  const R ql1 = -qm1 + (R)5 * qc + (R)2 * qp1;
  const R ql2 = (R)2 * qm2 - (R)7 * qm1 + (R)11 * qc;
  const R qr0 = (R)11 * qc - (R)7 * qp1 + (R)2 * qp2;
  const R qr1 = (R)2 * qm1 + (R)5 * qc - qp1;
  const R qr2 = -qm2 + (R)5 * qm1 + (R)2 * qc;
  const R numl = nl0 * ql0 + nl1 * ql1 + nl2 * ql2, denl = (R)6 * (nl0 + nl1 + nl2);
  const R numr = nr0 * qr0 + nr1 * qr1 + nr2 * qr2, denr = (R)6 * (nr0 + nr1 + nr2);
  if (sizeof(R) == 8) {
    // one reciprocal for both (the product stays far inside double range)
    const R inv = (R)1 / (denl * denr);
    L = numl * denr * inv;
    Rr = numr * denl * inv;
  } else {
#ifdef __CUDA_ARCH__
    L = __fdividef((float)numl, (float)denl);
    Rr = __fdividef((float)numr, (float)denr);
#else
    L = (float)numl / (float)denl;
    Rr = (float)numr / (float)denr;
#endif
  }
}

// weno_lr of two quantities in FP64 with one reciprocal for the four face
// values (the product of the four denominators stays inside double range:
// each lies between about 6e-24 and 1e40 for |q| below 1e4)
VH_HD inline void weno_lr_pair(const double* a, const double* b, double& La, double& Ra, double& Lb, double& Rb) {
  double num[4], den[4];
  const double* q[2] = {a, b};
  for (int m = 0; m < 2; m++) {
    const double qm2 = q[m][0], qm1 = q[m][1], qc = q[m][2], qp1 = q[m][3], qp2 = q[m][4];
    double b0, b1, b2;
    weno_beta<double>(qm2, qm1, qc, qp1, qp2, b0, b1, b2);
    const double eps = 1e-6;
    const double e0 = eps + b0, e1 = eps + b1, e2 = eps + b2;
    const double E0 = e0 * e0, E1 = e1 * e1, E2 = e2 * e2;
    const double P12 = E1 * E2, P02 = E0 * E2, P01 = E0 * E1;
    const double nl0 = 0.3 * P12, nl1 = 0.6 * P02, nl2 = 0.1 * P01;
    const double nr0 = 0.1 * P12, nr1 = nl1, nr2 = 0.3 * P01;
    const double ql0 = 2 * qc + 5 * qp1 - qp2;
    const double ql1 = -qm1 + 5 * qc + 2 * qp1;
    const double ql2 = 2 * qm2 - 7 * qm1 + 11 * qc;
    const double qr0 = 11 * qc - 7 * qp1 + 2 * qp2;
    const double qr1 = 2 * qm1 + 5 * qc - qp1;
    const double qr2 = -qm2 + 5 * qm1 + 2 * qc;
    num[2 * m] = nl0 * ql0 + nl1 * ql1 + nl2 * ql2;
    den[2 * m] = 6 * (nl0 + nl1 + nl2);
    num[2 * m + 1] = nr0 * qr0 + nr1 * qr1 + nr2 * qr2;
    den[2 * m + 1] = 6 * (nr0 + nr1 + nr2);
  }
  const double d01 = den[0] * den[1], d23 = den[2] * den[3];
  const double inv = 1.0 / (d01 * d23);
  const double i01 = d23 * inv, i23 = d01 * inv;  // 1/(den0 den1), 1/(den2 den3)
  La = num[0] * den[1] * i01;
  Ra = num[1] * den[0] * i01;
  Lb = num[2] * den[3] * i23;
  Rb = num[3] * den[2] * i23;
}

// generalized minmod (theta) piecewise-linear face values (utils.h:33-55)
template <class R>
VH_HD inline R mm3(R a, R b, R c) {
  if (a * b > (R)0 && b * c > (R)0) {
    R m = fmin(fmin(fabs(a), fabs(b)), fabs(c));
    return a < (R)0 ? -m : m;
  }
  return (R)0;
}
template <class R>
VH_HD inline R mm_left(R th, R qm1, R qc, R qp1) {
  return qc + (R)0.5 * mm3<R>(th * (qc - qm1), (R)0.5 * (qp1 - qm1), th * (qp1 - qc));
}
template <class R>
VH_HD inline R mm_right(R th, R qm1, R qc, R qp1) {
  return qc - (R)0.5 * mm3<R>(th * (qc - qm1), (R)0.5 * (qp1 - qm1), th * (qp1 - qc));
}

// --------------------------------------------------------------- IS source
// Shear, expansion and acceleration at one cell, then the source of the five
// evolved pi components in the flux form d_tau pi + d_i(v^i pi) = S:
//   S = [ -(pi - 2 eta sigma)/taupi - (4/3) pi theta
//         - (u^mu pi^{nu b} + u^nu pi^{mu b}) a_b
//         - u^a (Gamma^mu_{a l} pi^{l nu} + Gamma^nu_{a l} pi^{mu l}) ] / u^tau
//       + pi d_i v^i
// with sigma the fully projected shear tensor, theta = nabla.u and
// a_b = u^a nabla_a u_b (NEWEST5/Source.h:317-370; Cartesian: no
// Christoffels, TXYZ5/Source.h:291-335).  du[l][m] = d_m u^l.  The step
// needs the rows x and y of sigma (columns x, y, eta); FULL fills all of it.
template <class R, bool FULL = false>
VH_HD inline void is_kinematics(int cart, R tau, const R* u, const R du[4][4], R sig[4][4], R& theta, R acc[4]) {
  const R t2 = cart ? (R)1 : tau * tau;
  const R g[4] = {(R)1, (R)-1, (R)-1, -t2};
  const R gi[4] = {(R)1, (R)-1, (R)-1, cart ? (R)-1 : (R)-1 / t2};
  R Dm[4][4];
#pragma unroll
  for (int l = 0; l < 4; l++)
#pragma unroll
    for (int a = 0; a < 4; a++) Dm[l][a] = du[l][a];
  if (!cart) {
    const R itau = (R)1 / tau;
    Dm[0][3] += tau * u[3];
    Dm[3][0] += u[3] * itau;
    Dm[3][3] += u[0] * itau;
  }
  R Dl[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) Dl[a][b] = g[b] * Dm[b][a];
  theta = Dm[0][0] + Dm[1][1] + Dm[2][2] + Dm[3][3];
  R Dt[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) Dt[a][b] = (a == b ? gi[a] : (R)0) - u[a] * u[b];
  R tr = 0;
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) tr += Dt[a][b] * Dl[a][b];
  const R tr3 = tr * ((R)1 / (R)3);
  R S[4][4], M[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) S[a][b] = (R)0.5 * (Dl[a][b] + Dl[b][a]);
  // the step uses only sigma^{xx}, sigma^{yy}, sigma^{xy}, sigma^{x eta},
  // sigma^{y eta} (rows x, y and columns x, y, eta)
  constexpr int m0 = FULL ? 0 : 1, m1 = FULL ? 4 : 3, v0 = FULL ? 0 : 1;
#pragma unroll
  for (int m = m0; m < m1; m++)
#pragma unroll
    for (int b = 0; b < 4; b++) {
      R s = 0;
#pragma unroll
      for (int a = 0; a < 4; a++) s += Dt[m][a] * S[a][b];
      M[m][b] = s;
    }
#pragma unroll
  for (int m = m0; m < m1; m++)
#pragma unroll
    for (int v = v0; v < 4; v++) {
      R s = 0;
#pragma unroll
      for (int b = 0; b < 4; b++) s += M[m][b] * Dt[v][b];
      sig[m][v] = s - Dt[m][v] * tr3;
    }
#pragma unroll
  for (int v = 0; v < 4; v++) {
    R s = 0;
#pragma unroll
    for (int a = 0; a < 4; a++) s += u[a] * Dm[v][a];
    acc[v] = g[v] * s;
  }
}

// the shear source with P(e) and T(e) already known
template <class R>
VH_HD inline void is_source_PT(const DevCfg& C, R tau, R e, R P, R T, const R* u, const R* p, const R du[4][4],
                               R out[5]) {
  const int cart = C.cart;
  const R t2 = cart ? (R)1 : tau * tau;
  R eta, tp;
  transport_T<R>(C, e, P, T, &eta, &tp);
  PiDep<R> d = pi_dep<R>(u[0], u[1], u[2], u[3], p, t2);
  R pi[4][4] = {{d.tt, d.tx, d.ty, d.te}, {d.tx, p[0], p[2], p[3]}, {d.ty, p[2], p[1], p[4]}, {d.te, p[3], p[4], d.ee}};
  R sig[4][4], th, acc[4];
  is_kinematics<R>(cart, tau, u, du, sig, th, acc);
  R pa[4];
#pragma unroll
  for (int v = 0; v < 4; v++) pa[v] = pi[v][0] * acc[0] + pi[v][1] * acc[1] + pi[v][2] * acc[2] + pi[v][3] * acc[3];
  const R iu0 = (R)1 / u[0], itp = (R)1 / tp, itau = cart ? (R)1 : (R)1 / tau;
  R divv = 0;
#pragma unroll
  for (int i = 1; i < 4; i++) divv += du[i][i] * iu0 - u[i] * du[0][i] * (iu0 * iu0);
  const int MU[5] = {1, 2, 1, 1, 2}, NU[5] = {1, 2, 2, 3, 3};
#pragma unroll
  for (int q = 0; q < 5; q++) {
    const int m = MU[q], v = NU[q];
    const R relax = C.cold ? (R)0 : pi[m][v];  // the cold-plasma limit keeps 2 eta sigma / tau_pi only
    R rhs = -(relax - (R)2 * eta * sig[m][v]) * itp - ((R)4 / (R)3) * pi[m][v] * th - (u[m] * pa[v] + u[v] * pa[m]);
    R chr = 0;
    if (!cart) {
#pragma unroll
      for (int w = 0; w < 2; w++) {
        const int Aa = w ? v : m, Bb = w ? m : v;
        if (Aa == 0) chr += u[3] * tau * pi[3][Bb];
        if (Aa == 3) chr += (u[0] * pi[3][Bb] + u[3] * pi[0][Bb]) * itau;
      }
    }
    out[q] = (rhs - chr) * iu0 + pi[m][v] * divv;
  }
}

template <class R>
VH_HD inline void is_source(const DevCfg& C, R tau, R e, const R* u, const R* p, const R du[4][4], R out[5]) {
  R P, cs2, T;
  eos_all<R>(C, e, P, cs2, T);
  is_source_PT<R>(C, tau, e, P, T, u, p, du, out);
}

// P and dP/de together (one table lookup)
template <class R>
VH_HD inline void eos_P_cs2(const DevCfg& C, R e, R& P, R& cs2) {
  if (C.eos_kind == 0) { P = e / (R)3; cs2 = (R)1 / (R)3; return; }
  R T;
  eos_table<R>(C, e, &P, &cs2, &T);
}

// -------------------------------------------------------------- con2prim
// Residuals of T^{tau nu} u_nu = e u^tau for x = (e, u^x, u^y, u^eta) and
// their Jacobian (NEWEST5/multiroot.h:202-319), in double.
VH_HD inline void c2p_fj(const DevCfg& C, const double* Tt, const double* p, double t2, const double* x,
                              double* y, double J[4][4], bool jac) {
  double e = x[0];
  const double u1 = x[1], u2 = x[2], u3 = x[3];
  if (e <= 0) e = 1e-6;  // NEWEST5/multiroot.h:225-226
  double P, a;
  eos_P_cs2<double>(C, e, P, a);
  const double W = Tt[0], X = Tt[1], Y = Tt[2], Z = Tt[3];
  const double p1 = p[0], p2 = p[1], p3 = p[2], p4 = p[3], p5 = p[4];
  const double S = 1 + u1 * u1 + u2 * u2 + t2 * u3 * u3;
  const double u0 = sqrt(S);
  const double ep = e + P;
  y[0] = (W - e) * u0 - X * u1 - Y * u2 - t2 * Z * u3;
  y[1] = X * u0 - e * u1 - u1 * (P + p1 + ep * u1 * u1) - u2 * (p3 + ep * u1 * u2) - t2 * u3 * (p4 + ep * u1 * u3);
  y[2] = Y * u0 - e * u2 - u1 * (p3 + ep * u1 * u2) - u2 * (P + p2 + ep * u2 * u2) - t2 * u3 * (p5 + ep * u2 * u3);
  y[3] = Z * u0 - p4 * u1 - p5 * u2 - u3 * (P + W - p1 - p2);
  if (!jac) return;
  const double iu = 1.0 / u0;
  J[0][0] = -u0;
  J[0][1] = (W - e) * u1 * iu - X;
  J[0][2] = (W - e) * u2 * iu - Y;
  J[0][3] = t2 * ((W - e) * u3 * iu - Z);
  J[1][0] = -(1 + a) * u1 * S;
  J[1][1] = X * u1 * iu - p1 - ep * (1 + 3 * u1 * u1 + u2 * u2 + t2 * u3 * u3);
  J[1][2] = X * u2 * iu - p3 - 2 * ep * u1 * u2;
  J[1][3] = t2 * (X * u3 * iu - p4 - 2 * ep * u1 * u3);
  J[2][0] = -(1 + a) * u2 * S;
  J[2][1] = Y * u1 * iu - p3 - 2 * ep * u1 * u2;
  J[2][2] = Y * u2 * iu - p2 - ep * (1 + u1 * u1 + 3 * u2 * u2 + t2 * u3 * u3);
  J[2][3] = t2 * (Y * u3 * iu - p5 - 2 * ep * u2 * u3);
  J[3][0] = -a * u3;
  J[3][1] = Z * u1 * iu - p4;
  J[3][2] = Z * u2 * iu - p5;
  J[3][3] = t2 * Z * u3 * iu - (P + W - p1 - p2);
}

// Gaussian elimination with partial pivoting on a 4x4 system (in place).
// Row swaps are written as compile-time-indexed selects so that the matrix
// stays in registers.
VH_HD inline bool solve4(double A[4][4], double b[4]) {
#pragma unroll
  for (int c = 0; c < 4; c++) {
    int p = c;
    double best = fabs(A[c][c]);
#pragma unroll
    for (int r = c + 1; r < 4; r++)
      if (fabs(A[r][c]) > best) { best = fabs(A[r][c]); p = r; }
    if (best == 0.0) return false;
#pragma unroll
    for (int r = c + 1; r < 4; r++) {
      if (r == p) {
#pragma unroll
        for (int k = 0; k < 4; k++) { double t = A[c][k]; A[c][k] = A[r][k]; A[r][k] = t; }
        double t = b[c]; b[c] = b[r]; b[r] = t;
      }
    }
    const double ip = 1.0 / A[c][c];
    A[c][c] = ip;  // keep the reciprocal pivot for the back substitution
#pragma unroll
    for (int r = c + 1; r < 4; r++) {
      const double m = A[r][c] * ip;
#pragma unroll
      for (int k = c + 1; k < 4; k++) A[r][k] -= m * A[c][k];
      b[r] -= m * b[c];
    }
  }
#pragma unroll
  for (int c = 3; c >= 0; c--) {
    double s = b[c];
#pragma unroll
    for (int k = c + 1; k < 4; k++) s -= A[c][k] * b[k];
    b[c] = s * A[c][c];
  }
  return true;
}

// Newton with norm-reducing step control and the reference's form of
// stopping rule (|dx_i| < rtol |x_i| or dx_i = 0 for all i, at most 100
// iterations; NEWEST5/multiroot.h:389-422, where rtol = 1e-16).  A step that
// raises |f| is shortened by t = (sqrt(1+6r)-1)/(3r), r = |f_new|^2/|f_old|^2,
// at most 64 times.  Returns the iteration count, or -1 on failure.
// The step stops at rtol = 1e-13 in FP64 and 1e-10 in the mixed mode (which
// stores the result in single precision).  Newton converges quadratically,
// so an iterate reached by a step below 1e-13 relative is the root to
// rounding; the reference's 1e-16 mostly waits for steps that round to zero
// (about 1.5 more iterations per cell, and warps wait for their slowest
// cell).  The Jacobian is formed together with the residual at every trial
// point, so an accepted full step (the common case) costs one evaluation.
// With qtol > 0 the loop also stops after an undamped step with every
// |dx_i| <= qtol |x_i| (or dx_i = 0): in the quadratic regime the error left
// after such a step is of order |dx|^2, so qtol = 1e-8 leaves ~1e-16 and
// saves the confirming iteration whose step would fall below rtol.
// With qskip > 0 a Newton step whose every component is already below
// qskip |x_i + st_i| (or zero) is taken without evaluating the residual at
// its end: that evaluation would only confirm, through the step control, a
// step of a size that the quadratic regime always accepts, so the iterate
// is the one the loop above would reach (one evaluation fewer per cell,
// the last of three or four).  The root test then applies to the residual
// before that step, against fskip |T^{tau mu}|: a Newton step of relative
// size qskip leaves a residual of about qskip |J x|.
VH_HD inline int con2prim(const DevCfg& C, const double* Tt, const double* p, double tau, double* x,
                               double rtol = 1e-16, double qtol = 0.0, double qskip = 0.0, double fskip = 0.0) {
  const double t2 = C.cart ? 1.0 : tau * tau;
  double y[4], J[4][4];
  c2p_fj(C, Tt, p, t2, x, y, J, true);
  // squared residual norms: the step control compares and divides squares,
  // so no square root is taken per trial point
  double phi = y[0] * y[0] + y[1] * y[1] + y[2] * y[2] + y[3] * y[3];
  int it = 0;
  while (it < 100) {
    it++;
    double st[4] = {-y[0], -y[1], -y[2], -y[3]};
    if (!solve4(J, st)) return -1;
    if (qskip > 0.0) {
      bool small = true;
#pragma unroll
      for (int i = 0; i < 4; i++)
        if (!(fabs(st[i]) <= qskip * fabs(x[i] + st[i]) || st[i] == 0.0)) small = false;
      if (small) {
#pragma unroll
        for (int i = 0; i < 4; i++) x[i] += st[i];
        const double sc = fskip * (fabs(Tt[0]) + fabs(Tt[1]) + fabs(Tt[2]) + fabs(Tt[3]));
        return phi <= sc * sc ? it : -1;
      }
    }
    double t = 1.0, xt[4], phi1 = 0;
    bool ok = false;
    for (int tries = 0; tries < 64; tries++) {
#pragma unroll
      for (int i = 0; i < 4; i++) xt[i] = x[i] + t * st[i];
      c2p_fj(C, Tt, p, t2, xt, y, J, true);
      if (!(isfinite(y[0]) && isfinite(y[1]) && isfinite(y[2]) && isfinite(y[3]))) return -1;
      phi1 = y[0] * y[0] + y[1] * y[1] + y[2] * y[2] + y[3] * y[3];
      if (phi1 <= phi || phi == 0.0) { ok = true; break; }
      const double r = phi1 / phi;
      t *= (sqrt(1.0 + 6.0 * r) - 1.0) / (3.0 * r);
    }
    if (!ok) return -1;
    bool conv = true, quad = t == 1.0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      double dx = xt[i] - x[i];
      x[i] = xt[i];
      if (!(fabs(dx) < rtol * fabs(x[i]) || dx == 0.0)) conv = false;
      if (!(fabs(dx) <= qtol * fabs(x[i]) || dx == 0.0)) quad = false;
    }
    if (quad) conv = true;
    phi = phi1;
    if (conv) break;
  }
  // an iterate that is not a root is a failure (the reference keeps it
  // silently after 100 iterations): residual above 1e-8 of |T^{tau mu}|
  const double scale = 1e-8 * (fabs(Tt[0]) + fabs(Tt[1]) + fabs(Tt[2]) + fabs(Tt[3]));
  if (!(phi <= scale * scale)) return -1;
  return it;
}

}  // namespace vh
