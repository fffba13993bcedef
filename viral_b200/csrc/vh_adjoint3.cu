// Discrete adjoint of the viscous KT step on 3+1D Milne grids (WENO5, copy
// boundaries): gradients of the momentum anisotropy
// eps_p = sum(T^xx - T^yy) / sum(T^xx + T^yy) over every interior cell at the
// final time, with respect to the initial state (all 18 fields) and to the
// eta/s(T) parameters.  The scheme is the boost-invariant adjoint's
// (vh_adjoint.cu) with every field evolved: u^eta, pi^{x eta}, pi^{y eta},
// T^{tau eta}, the eta sweep and its line adjoints, the eta Christoffel terms
// of the sources and the four-unknown root-find.
//   k_adj3_stage2  per interior cell: ghost images folded in, the root of
//                  stage 2 by the implicit-function theorem, the RK2 average,
//                  the sources at tau_{n+1} and du/dtau
//   k_adj3_dir     one block per line along x, y or eta: the KT fluxes, WENO
//                  face states and velocity derivatives of the stage in
//                  reverse
//   k_adj3_stage1  as k_adj3_stage2 for stage 1 (sources at tau_n)
// Every adjoint is written by exactly one thread (no atomics), so the
// gradient is deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "vh.h"
#include "vh_adjoint3.cuh"
#include "vh_adjoint_run.cuh"
#include "vh_handle.cuh"
#include "vh_nvtx.h"

namespace {

using namespace vh;

constexpr int NXO3 = NX3 + 4;  // own adjoint of X: the 14 cell variables and prevu
constexpr int X3PU = NX3;
constexpr int REC3_X = 0, REC3_Y = 1;
constexpr int kRecY3 = 14;  // Y record: e, u^mu, the stage-1 conserved set (T^{tau mu}, pi)
constexpr int NVEL = 4;     // velocity lines of the WENO derivatives (u^tau .. u^eta)
constexpr int KQ3 = NQ3 + NVEL;
enum : unsigned { AST3_SINGULAR = 1u };

// the 14 cell variables of a record at cell c
template <class R>
__device__ __forceinline__ void load_cell3(const R* rec, int kind, long long n, long long c, R* x) {
  x[X3E] = rec[c];
#pragma unroll
  for (int l = 0; l < 4; l++) x[X3U + l] = rec[(1 + l) * n + c];
  if (kind == REC3_X) {
#pragma unroll
    for (int l = 0; l < 5; l++) x[X3P + l] = rec[(5 + l) * n + c];
#pragma unroll
    for (int l = 0; l < 4; l++) x[X3T + l] = rec[(10 + l) * n + c];
  } else {
#pragma unroll
    for (int l = 0; l < 4; l++) x[X3T + l] = rec[(5 + l) * n + c];
#pragma unroll
    for (int l = 0; l < 5; l++) x[X3P + l] = rec[(9 + l) * n + c];
  }
}

// WENO velocity derivatives along x, y and eta at an interior cell, as the
// flux sweeps compute them: du[l][1 + d] for u^l (U points at u^tau)
template <class R>
__device__ __forceinline__ void du_space3(const DevCfg& C, const R* U, long long n, long long c, R du[4][4]) {
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const long long s = d == 0 ? 1 : (d == 1 ? (long long)C.px : (long long)C.px * C.gy);
    const R inv_h = (R)(1.0 / (d == 0 ? C.dx : (d == 1 ? C.dy : C.dz)));
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const R* q = U + l * n + c;
      R L, Rr;
      weno_lr<R>(q[-2 * s], q[-s], q[0], q[s], q[2 * s], L, Rr);
      du[l][1 + d] = (L - Rr) * inv_h;
    }
  }
}

// the face ghost cells that the forward fills from interior cell (i, j, k)
template <class F>
__device__ __forceinline__ void for_images3(const DevCfg& C, int i, int j, int k, F&& f) {
  if (i == C.il)
    for (int m = 0; m < NG; m++) f(cix(C, m, j, k));
  if (i == C.ir - 1)
    for (int m = 0; m < NG; m++) f(cix(C, C.ir + m, j, k));
  if (j == C.jl)
    for (int m = 0; m < NG; m++) f(cix(C, i, m, k));
  if (j == C.jr - 1)
    for (int m = 0; m < NG; m++) f(cix(C, i, C.jr + m, k));
  if (k == C.kl)
    for (int m = 0; m < NG; m++) f(cix(C, i, j, m));
  if (k == C.kr - 1)
    for (int m = 0; m < NG; m++) f(cix(C, i, j, C.kr + m));
}

template <class R>
struct Adj3Args {
  DevCfg C;
  long long n;
  const R* X;    // record X_n
  const R* Y;    // record Y_n
  const R* X1;   // record X_{n+1}
  R* xo;         // own adjoint of X: 18 fields
  R* xd;         // line adjoints of X: 3 x 14 fields (x, y, eta lines)
  R* yo;         // own adjoint of Y: 14 fields
  R* yd;         // line adjoints of Y: 3 x 14 fields
  R* resb;       // 9: adjoint of the flux divergence (T^{tau mu}, pi)
  R* dub;        // 12: adjoint of du^l/dx^d at (l*3 + d)
  R* v1tb;       // 4: adjoint of the stage-1 tau T^{tau mu}
  double* cacc;  // 2 per cell: d/d(etas0, etas1)
  unsigned* status;
  double tau_n, ts;
};

// the own and line adjoints of a recorded state at interior cell c, with
// the adjoints of its ghost images (copies of the cell) folded in
template <class R>
__device__ __forceinline__ void gather3(const Adj3Args<R>& a, const R* own, const R* line, int i, int j, int k,
                                        long long c, R* v) {
  const long long n = a.n;
#pragma unroll
  for (int f = 0; f < NX3; f++)
    v[f] = own[f * n + c] + line[f * n + c] + line[(NX3 + f) * n + c] + line[(2 * NX3 + f) * n + c];
  for_images3(a.C, i, j, k, [&](long long g) {
#pragma unroll
    for (int f = 0; f < NX3; f++) v[f] += line[f * n + g] + line[(NX3 + f) * n + g] + line[(2 * NX3 + f) * n + g];
  });
}

// adjoint of the root (e, u^x, u^y, u^eta; u^tau follows) -> adjoint of the
// conserved set it came from, added to the direct adjoints of that set
template <class R>
__device__ __forceinline__ void root_adjoint3(const Adj3Args<R>& a, const R* rec, int kind, long long c,
                                              double tau1, const R* v, R* Tt, R* Pp) {
  R x[NX3];
  load_cell3<R>(rec, kind, a.n, c, x);
  const double t2 = tau1 * tau1;
  const double u0 = x[X3U], u1 = x[X3U + 1], u2 = x[X3U + 2], u3 = x[X3U + 3];
  const double u0b = v[X3U];
  const double xb[4] = {(double)v[X3E], (double)v[X3U + 1] + u0b * u1 / u0, (double)v[X3U + 2] + u0b * u2 / u0,
                        (double)v[X3U + 3] + u0b * t2 * u3 / u0};
  double T4[4], p5[5];
#pragma unroll
  for (int l = 0; l < 4; l++) T4[l] = x[X3T + l];
#pragma unroll
  for (int l = 0; l < 5; l++) p5[l] = x[X3P + l];
  const double x4[4] = {(double)x[X3E], u1, u2, u3};
  double Tb[4] = {0, 0, 0, 0}, pb[5] = {0, 0, 0, 0, 0};
  if (!c2p_ift_vjp4(a.C, T4, p5, tau1, x4, xb, Tb, pb)) atomicOr(a.status, AST3_SINGULAR);
#pragma unroll
  for (int l = 0; l < 4; l++) Tt[l] = v[X3T + l] + (R)Tb[l];
#pragma unroll
  for (int l = 0; l < 5; l++) Pp[l] = v[X3P + l] + (R)pb[l];
}

// writes a stage's divergence and gradient adjoints and the parameter sums
template <class R>
__device__ __forceinline__ void put_stage(const Adj3Args<R>& a, long long c, const R* rb, const R dub[4][4],
                                          const R* cb) {
  const long long n = a.n;
#pragma unroll
  for (int q = 0; q < 9; q++) a.resb[q * n + c] = rb[q];
#pragma unroll
  for (int l = 0; l < 4; l++)
#pragma unroll
    for (int d = 0; d < 3; d++) a.dub[(l * 3 + d) * n + c] = dub[l][1 + d];
  a.cacc[c] += (double)cb[0];
  a.cacc[n + c] += (double)cb[1];
}

// Reverse of stage 2 of step n at every interior cell.
template <class R>
__global__ void __launch_bounds__(128) k_adj3_stage2(Adj3Args<R> a) {
  const DevCfg& C = a.C;
  const long long n = a.n;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)C.nx * C.ny * C.nz) return;
  const CellAt at = cell_at(C, t);
  const long long c = at.c;
  const double tau1 = a.tau_n + a.ts;
  const R ts = (R)a.ts;

  R v[NX3];
  gather3<R>(a, a.xo, a.xd, at.i, at.j, at.k, c, v);
  R VT[4], Vp[5];
  root_adjoint3<R>(a, a.X1, REC3_X, c, tau1, v, VT, Vp);
#pragma unroll
  for (int l = 0; l < 4; l++) VT[l] = VT[l] / (R)tau1;  // A' = Vn / tau1 (T part)

  // Vn = 1/2 tau_n A + 1/2 v1t + 1/2 ts (res + src)   (T^{tau mu})
  //      1/2 A + 1/2 B + 1/2 ts (res + src)           (pi)
  R xn[NXO3], yb[NX3], rb[9];
#pragma unroll
  for (int f = 0; f < NXO3; f++) xn[f] = 0;
#pragma unroll
  for (int f = 0; f < NX3; f++) yb[f] = 0;
  const R half = (R)0.5;
#pragma unroll
  for (int l = 0; l < 4; l++) {
    xn[X3T + l] = half * (R)a.tau_n * VT[l];
    a.v1tb[l * n + c] = half * VT[l];
    rb[l] = half * ts * VT[l];
  }
#pragma unroll
  for (int l = 0; l < 5; l++) {
    xn[X3P + l] = half * Vp[l];
    yb[X3P + l] = half * Vp[l];
    rb[4 + l] = half * ts * Vp[l];
  }
  // sources at tau_{n+1} from Y_n; du/dtau = (u(Y) - u(X)) / ts
  R y[NX3];
  load_cell3<R>(a.Y, REC3_Y, n, c, y);
  R du[4][4];
#pragma unroll
  for (int l = 0; l < 4; l++) du[l][0] = (y[X3U + l] - a.X[(1 + l) * n + c]) / ts;
  du_space3<R>(C, a.Y + n, n, c, du);
  R eb = 0, ub[4] = {0, 0, 0, 0}, pb[5] = {0, 0, 0, 0, 0}, dub[4][4] = {}, cb[2] = {0, 0};
  src3_vjp<R>(C, (R)tau1, y[X3E], y + X3U, y + X3P, du, rb, eb, ub, pb, dub, cb);
  yb[X3E] += eb;
#pragma unroll
  for (int l = 0; l < 4; l++) {
    yb[X3U + l] += ub[l] + dub[l][0] / ts;
    xn[X3U + l] += a.xo[(X3PU + l) * n + c] - dub[l][0] / ts;  // prevu of X_{n+1} is u of X_n
  }
#pragma unroll
  for (int l = 0; l < 5; l++) yb[X3P + l] += pb[l];
#pragma unroll
  for (int f = 0; f < NXO3; f++) a.xo[f * n + c] = xn[f];
#pragma unroll
  for (int f = 0; f < NX3; f++) a.yo[f * n + c] = yb[f];
  put_stage<R>(a, c, rb, dub, cb);
}

// Reverse of stage 1 of step n at every interior cell.
template <class R>
__global__ void __launch_bounds__(128) k_adj3_stage1(Adj3Args<R> a) {
  const DevCfg& C = a.C;
  const long long n = a.n;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)C.nx * C.ny * C.nz) return;
  const CellAt at = cell_at(C, t);
  const long long c = at.c;
  const double tau1 = a.tau_n + a.ts;
  const R ts = (R)a.ts;

  R w[NX3];
  gather3<R>(a, a.yo, a.yd, at.i, at.j, at.k, c, w);
  R VT[4], Vp[5];
  root_adjoint3<R>(a, a.Y, REC3_Y, c, tau1, w, VT, Vp);
#pragma unroll
  for (int l = 0; l < 4; l++) VT[l] = VT[l] / (R)tau1 + a.v1tb[l * n + c];  // B = Vn / tau1, v1t = Vn

  // Vn = tau_n A + ts (res + src)   (T^{tau mu});   A + ts (res + src)   (pi)
  R xn[NXO3], rb[9];
#pragma unroll
  for (int f = 0; f < NXO3; f++) xn[f] = a.xo[f * n + c];
#pragma unroll
  for (int l = 0; l < 4; l++) {
    xn[X3T + l] += (R)a.tau_n * VT[l];
    rb[l] = ts * VT[l];
  }
#pragma unroll
  for (int l = 0; l < 5; l++) {
    xn[X3P + l] += Vp[l];
    rb[4 + l] = ts * Vp[l];
  }
  R x[NX3];
  load_cell3<R>(a.X, REC3_X, n, c, x);
  R du[4][4];
#pragma unroll
  for (int l = 0; l < 4; l++) du[l][0] = (x[X3U + l] - a.X[(14 + l) * n + c]) / ts;
  du_space3<R>(C, a.X + n, n, c, du);
  R eb = 0, ub[4] = {0, 0, 0, 0}, pb[5] = {0, 0, 0, 0, 0}, dub[4][4] = {}, cb[2] = {0, 0};
  src3_vjp<R>(C, (R)a.tau_n, x[X3E], x + X3U, x + X3P, du, rb, eb, ub, pb, dub, cb);
  xn[X3E] += eb;
#pragma unroll
  for (int l = 0; l < 4; l++) {
    xn[X3U + l] += ub[l] + dub[l][0] / ts;
    xn[X3PU + l] -= dub[l][0] / ts;
  }
#pragma unroll
  for (int l = 0; l < 5; l++) xn[X3P + l] += pb[l];
#pragma unroll
  for (int f = 0; f < NXO3; f++) a.xo[f * n + c] = xn[f];
  put_stage<R>(a, c, rb, dub, cb);
}

template <class R>
struct Dir3Args {
  DevCfg C;
  long long n;
  const R* rec;  // recorded primal state of the stage
  int kind;      // REC3_X or REC3_Y
  R tau_s;       // time the stage's fluxes were formed at
  const R* resb;
  const R* dub;
  R* out;        // 3 x 14 fields: line adjoints (x lines, y lines, eta lines)
};

// quantities whose WENO stencils are reversed at the same time, and
// shared-memory words per line cell: flux quantities 19, flux adjoints 9,
// max speed 1, speed-state adjoints 2, quantity adjoints 23, velocities 4,
// and one region used first for the face states (2 x 10) and then for the
// stencil contributions (5 per quantity in flight)
constexpr int kQP3 = 4;
constexpr int kDir3Shared = 5 * kQP3 > 20 ? 5 * kQP3 : 20;
constexpr int kDir3Words = NQ3 + 9 + 1 + 2 + KQ3 + NVEL + kDir3Shared;

template <class R>
__device__ __forceinline__ R sgn3(R x) { return (R)((x > (R)0) - (x < (R)0)); }

// Reverse of the flux sweep of one stage along one line (the whole line,
// interior and both ghost layers, in shared memory).
template <class R, int DIR>
__device__ __forceinline__ void adj_line3(const Dir3Args<R>& a, int line, R* sm) {
  const DevCfg& C = a.C;
  const long long n = a.n;
  const int G = DIR == 0 ? C.gx : (DIR == 1 ? C.gy : C.gz);
  const int lo = DIR == 0 ? C.il : (DIR == 1 ? C.jl : C.kl), hi = DIR == 0 ? C.ir : (DIR == 1 ? C.jr : C.kr);
  const long long stride = DIR == 0 ? 1 : (DIR == 1 ? (long long)C.px : (long long)C.px * C.gy);
  long long base;
  if (DIR == 0) base = cix(C, 0, C.jl + line % C.ny, C.kl + line / C.ny);
  else if (DIR == 1) base = cix(C, C.il + line % C.nx, 0, C.kl + line / C.nx);
  else base = cix(C, C.il + line % C.nx, C.jl + line / C.nx, 0);
  const double hh = DIR == 0 ? C.dx : (DIR == 1 ? C.dy : C.dz);
  const R h = (R)hh, inv_h = (R)(1.0 / hh);
  R* q = sm;              // 19: flux quantities
  R* hb = q + NQ3 * G;    // 9: adjoint of the KT flux at the face right of cell f
  R* am = hb + 9 * G;     // max signal speed at that face
  R* sl = am + G;         // adjoint of the speed's right-face state
  R* sr = sl + G;         // adjoint of the speed's left-face state
  R* qb = sr + G;         // 23: adjoints of the 19 quantities and of u^0..3
  R* uu = qb + KQ3 * G;   // 4: u^0..3 along the line
  R* lv = uu + NVEL * G;  // 10: face state at the right face (V^0..8, speed)
  R* rv = lv + 10 * G;    // 10: face state at the left face
  R* c5 = lv;             // 5 x kQP3: stencil contributions of the quantities in
                          // flight (after the face states are used)
  const int tid = threadIdx.x, nt = blockDim.x;

  for (int i = tid; i < G; i += nt) {
    R x[NX3], ql[NQ3];
    load_cell3<R>(a.rec, a.kind, n, base + i * stride, x);
    cell_q3<R, DIR>(C, a.tau_s, x, i >= lo && i < hi, ql);
#pragma unroll
    for (int k = 0; k < NQ3; k++) q[k * G + i] = ql[k];
#pragma unroll
    for (int l = 0; l < NVEL; l++) uu[l * G + i] = x[X3U + l];
#pragma unroll
    for (int k = 0; k < KQ3; k++) qb[k * G + i] = 0;
    sl[i] = 0;
    sr[i] = 0;
  }
  __syncthreads();
  const int ns = hi - lo + 2;  // cells lo-1 .. hi have full stencils
  for (int w = tid; w < 10 * ns; w += nt) {
    const int k = w / ns, i = lo - 1 + w % ns;
    const R* s = q + (9 + k) * G + i;
    weno_lr<R>(s[-2], s[-1], s[0], s[1], s[2], lv[k * G + i], rv[k * G + i]);
  }
  __syncthreads();
  // faces f | f+1 for f in [lo-1, hi-1]
  for (int f = lo - 1 + tid; f <= hi - 1; f += nt) {
    const long long cf = base + f * stride, cn = cf + stride;
    const R L = lv[9 * G + f], Rn = rv[9 * G + f + 1];
    const bool diss = f + 1 != lo;  // no dissipation left of the first interior cell
    const R amax = diss ? fmax(fabs(L), fabs(Rn)) : (R)0;
    R amb = 0;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const R rf = f >= lo ? a.resb[k * n + cf] : (R)0;
      const R rn = f + 1 < hi ? a.resb[k * n + cn] : (R)0;
      const R H = (rn - rf) * inv_h;  // res_i = -(H_{i+1/2} - H_{i-1/2}) / h
      hb[k * G + f] = H;
      amb -= (R)0.5 * (rv[k * G + f + 1] - lv[k * G + f]) * H;
    }
    am[f] = amax;
    if (diss) {
      if (fabs(L) >= fabs(Rn)) sl[f] = amb * sgn3(L);
      else sr[f + 1] = amb * sgn3(Rn);
    }
  }
  __syncthreads();
  // WENO stencils in reverse, kQP3 quantities at a time (the 19 flux
  // quantities, then the four velocity lines of the derivative du^l/dx^DIR)
  for (int k0 = 0; k0 < KQ3; k0 += kQP3) {
    for (int w = tid; w < kQP3 * G; w += nt) {
      const int kq = w / G, i = w % G, k = k0 + kq;
      R cc[5] = {0, 0, 0, 0, 0};
      if (k < KQ3 && i >= lo - 1 && i <= hi) {
        const bool hasL = i <= hi - 1, hasR = i >= lo;  // faces i and i-1
        R Lb = 0, Rb = 0;
        if (k < 9) {
          if (hasL) Lb = (R)0.5 * hb[k * G + i];
          if (hasR) Rb = (R)0.5 * hb[k * G + i - 1];
        } else if (k < 18) {
          if (hasL) Lb = (R)0.5 * am[i] * hb[(k - 9) * G + i];
          if (hasR) Rb = -(R)0.5 * am[i - 1] * hb[(k - 9) * G + i - 1];
        } else if (k == 18) {
          Lb = sl[i];
          Rb = sr[i];
        } else if (i >= lo && i < hi) {
          const R d = a.dub[((k - NQ3) * 3 + DIR) * n + base + i * stride];
          Lb = d / h;
          Rb = -d / h;
        }
        const R* s = k < NQ3 ? q + k * G : uu + (k - NQ3) * G;
        if (Lb != (R)0 || Rb != (R)0) weno_lr_vjp<R>(s + i - 2, Lb, Rb, cc);
      }
#pragma unroll
      for (int o = 0; o < 5; o++) c5[(kq * 5 + o) * G + i] = cc[o];
    }
    __syncthreads();
    for (int w = tid; w < kQP3 * G; w += nt) {
      const int kq = w / G, jj = w % G, k = k0 + kq;
      R acc = 0;
#pragma unroll
      for (int o = 0; o < 5; o++) {
        const int i = jj + 2 - o;
        if (i >= 0 && i < G) acc += c5[(kq * 5 + o) * G + i];
      }
      if (k < KQ3) qb[k * G + jj] += acc;
    }
    __syncthreads();
  }
  for (int jj = tid; jj < G; jj += nt) {
    const long long c = base + jj * stride;
    R x[NX3], qbl[NQ3], xb[NX3];
    load_cell3<R>(a.rec, a.kind, n, c, x);
#pragma unroll
    for (int k = 0; k < NQ3; k++) qbl[k] = qb[k * G + jj];
#pragma unroll
    for (int f = 0; f < NX3; f++) xb[f] = 0;
    cell_q3_vjp<R, DIR>(C, a.tau_s, x, jj >= lo && jj < hi, qbl, xb);
#pragma unroll
    for (int l = 0; l < NVEL; l++) xb[X3U + l] += qb[(NQ3 + l) * G + jj];
    R* out = a.out + (long long)DIR * NX3 * n;
#pragma unroll
    for (int f = 0; f < NX3; f++) out[f * n + c] = xb[f];
  }
}

// one block per line along DIR
template <class R, int DIR>
__global__ void __launch_bounds__(256) k_adj3_dir(Dir3Args<R> a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  adj_line3<R, DIR>(a, blockIdx.x, reinterpret_cast<R*>(smem_raw));
}

// line length, line count, threads and shared memory of the lines along d:
// 256 threads per line along x and y; along eta, where lines are short and
// many, the line length rounded up to warps (at most 256); shared memory for
// that line length only
struct LineShape {
  int G;
  long long lines;
  int threads;
  size_t smem;
};
template <class R>
LineShape line_shape(const DevCfg& C, int d) {
  LineShape s;
  s.G = d == 0 ? C.gx : (d == 1 ? C.gy : C.gz);
  s.lines = d == 0 ? (long long)C.ny * C.nz : (d == 1 ? (long long)C.nx * C.nz : (long long)C.nx * C.ny);
  s.threads = d == 2 ? std::min(256, (s.G + 31) / 32 * 32) : 256;
  s.smem = (size_t)kDir3Words * s.G * sizeof(R);
  return s;
}
template <class R>
size_t dir3_smem(const DevCfg& C) {
  return std::max(line_shape<R>(C, 0).smem, std::max(line_shape<R>(C, 1).smem, line_shape<R>(C, 2).smem));
}
template <class R>
int set_dir3_attrs(vh_handle* h) {
  VH_CUDA(h, cudaFuncSetAttribute(k_adj3_dir<R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)line_shape<R>(h->C, 0).smem));
  VH_CUDA(h, cudaFuncSetAttribute(k_adj3_dir<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)line_shape<R>(h->C, 1).smem));
  VH_CUDA(h, cudaFuncSetAttribute(k_adj3_dir<R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)line_shape<R>(h->C, 2).smem));
  return VH_OK;
}
// the reverse of one stage's three sweeps (independent: each writes its own
// line-adjoint plane)
template <class R>
int launch_dir3(vh_handle* h, const Dir3Args<R>& d) {
  const LineShape s0 = line_shape<R>(h->C, 0), s1 = line_shape<R>(h->C, 1), s2 = line_shape<R>(h->C, 2);
  k_adj3_dir<R, 0><<<(unsigned)s0.lines, s0.threads, s0.smem, h->stream>>>(d);
  k_adj3_dir<R, 1><<<(unsigned)s1.lines, s1.threads, s1.smem, h->stream>>>(d);
  k_adj3_dir<R, 2><<<(unsigned)s2.lines, s2.threads, s2.smem, h->stream>>>(d);
  VH_CUDA(h, cudaGetLastError());
  return VH_OK;
}

// adjoint seed: d eps_p / d (e, u^x, u^y, pi^xx, pi^yy) of the final state
template <class R>
__global__ void k_obs3_seed(DevCfg C, const R* S, long long n, const double* nd, R* xo) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)C.nx * C.ny * C.nz) return;
  const long long c = cell_at(C, t).c;
  R eb, u1b, u2b, p1b, p2b;
  obs_cell_vjp<R>(C, S[c], S[2 * n + c], S[3 * n + c], nd[0], nd[1], eb, u1b, u2b, p1b, p2b);
  xo[X3E * n + c] = eb;
  xo[(X3U + 1) * n + c] = u1b;
  xo[(X3U + 2) * n + c] = u2b;
  xo[X3P * n + c] = p1b;
  xo[(X3P + 1) * n + c] = p2b;
}

// gradients of the initial state: the 18 canonical fields (every field an
// independent variable) and the energy density of vh_init_profile (T^{tau mu}
// re-derived from e at fixed u and pi: T^{tau tau} = (e+P) u0^2 - P + pi^{tau
// tau}, T^{tau i} = (e+P) u0 u^i + pi^{tau i})
template <class R>
__global__ void k_adj3_final(DevCfg C, const R* X0, long long n, const R* xo, const R* xd, double* gs, double* ge) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  double v[NX3];
  for (int f = 0; f < NX3; f++)
    v[f] = (double)xo[f * n + c] + (double)xd[f * n + c] + (double)xd[(NX3 + f) * n + c] +
           (double)xd[(2 * NX3 + f) * n + c];
  if (gs) {
    gs[c] = v[X3E];
    for (int l = 0; l < 4; l++) {
      gs[(1 + l) * n + c] = v[X3U + l];
      gs[(10 + l) * n + c] = v[X3T + l];
      gs[(14 + l) * n + c] = (double)xo[(X3PU + l) * n + c];
    }
    for (int l = 0; l < 5; l++) gs[(5 + l) * n + c] = v[X3P + l];
  }
  if (ge) {
    double P, dP, T, dT;
    eos_d<double>(C, (double)X0[c], P, dP, T, dT);
    const double u0 = X0[n + c];
    double g = v[X3E] + v[X3T] * ((1 + dP) * u0 * u0 - dP);
    for (int l = 1; l < 4; l++) g += v[X3T + l] * (1 + dP) * u0 * (double)X0[(1 + l) * n + c];
    ge[c] = g;
  }
}

template <class R>
int adjoint3_run(vh_handle* h, const DevPtrs<R>& P, int nsteps, int every, double* eps_p, double* grad_state,
                 double* grad_e, double* grad_etas) {
  const DevCfg& C = h->C;
  const long long n = C.n;
  const size_t nb = (size_t)n * sizeof(R);
  cudaStream_t st = h->stream;
  const int nseg = (nsteps + every - 1) / every;
  const int seg_len = std::min(every, nsteps);
  // segments: the first takes the remainder, the others `every` steps each,
  // so the last one (recorded during the forward) is a full segment
  const int first = nsteps - (nseg - 1) * every;
  auto seg_start = [&](int k) { return k == 0 ? 0 : first + (k - 1) * every; };
  const int last0 = seg_start(nseg - 1);

  // ---- workspace (carved twice: once to size it, once to place it)
  struct Bufs {
    R *ck, *fin, *Xr, *Yr, *xo, *xd, *yo, *yd, *resb, *dub, *v1tb;
    double *cacc, *part, *nd, *sums, *gs, *ge;
    unsigned* ast;
  } B;
  auto layout = [&](Carve& c) {
    B.ck = c.take<R>((size_t)nseg * 18 * n);
    B.fin = c.take<R>((size_t)18 * n);
    B.Xr = c.take<R>((size_t)(seg_len + 1) * 18 * n);
    B.Yr = c.take<R>((size_t)seg_len * kRecY3 * n);
    B.xo = c.take<R>((size_t)NXO3 * n);
    B.xd = c.take<R>((size_t)3 * NX3 * n);
    B.yo = c.take<R>((size_t)NX3 * n);
    B.yd = c.take<R>((size_t)3 * NX3 * n);
    B.resb = c.take<R>((size_t)9 * n);
    B.dub = c.take<R>((size_t)12 * n);
    B.v1tb = c.take<R>((size_t)4 * n);
    B.cacc = c.take<double>((size_t)2 * n);
    B.part = c.take<double>((size_t)2 * kObsBlocks);
    B.nd = c.take<double>(2);
    B.sums = c.take<double>(2);
    B.ast = c.take<unsigned>(1);
    B.gs = c.take<double>((size_t)18 * n);
    B.ge = c.take<double>((size_t)n);
  };
  Carve cv;
  layout(cv);
  if (cv.off > h->adj_bytes) {
    VH_CUDA(h, cudaStreamSynchronize(st));
    cudaFree(h->adj_buf);
    h->adj_buf = nullptr;
    h->adj_bytes = 0;
    const cudaError_t e = cudaMalloc(&h->adj_buf, cv.off);
    if (e != cudaSuccess) {
      h->err = std::string("vh_adjoint_eps_p: workspace of ") + std::to_string(cv.off >> 20) +
               " MiB: " + cudaGetErrorString(e);
      return e == cudaErrorMemoryAllocation ? VH_E_NOMEM : VH_E_CUDA;
    }
    h->adj_bytes = cv.off;
  }
  Carve cw;
  cw.base = static_cast<char*>(h->adj_buf);
  layout(cw);
  if (int e = set_dir3_attrs<R>(h)) return e;
  PhaseClock clk;
  int t_start, t_fwd, t_end;
  VH_CUDA(h, clk.mark(st, &t_start));

  // ---- forward: a checkpoint at every segment start; the last segment is
  // recorded as it runs, so it is not recomputed
  const double ts = h->cfg.dtau;
  std::vector<double> taus(nsteps + 1);
  R* state = P.base0;
  int r;
  for (int s = 0; s < nsteps; s++) {
    if (s == 0 || (s >= first && (s - first) % every == 0)) {
      const int k = s == 0 ? 0 : (s - first) / every + 1;
      VH_CUDA(h, cudaMemcpyAsync(B.ck + (size_t)k * 18 * n, state, 18 * nb, cudaMemcpyDeviceToDevice, st));
    }
    taus[s] = h->tau;
    if (s >= last0)
      r = record_step<R>(h, P, B.Xr + (size_t)(s - last0) * 18 * n, B.Yr + (size_t)(s - last0) * kRecY3 * n);
    else
      r = step_once<R>(h, P);
    if (r) return r;
  }
  taus[nsteps] = h->tau;
  VH_CUDA(h, cudaMemcpyAsync(B.Xr + (size_t)(nsteps - last0) * 18 * n, state, 18 * nb, cudaMemcpyDeviceToDevice, st));
  VH_CUDA(h, cudaMemcpyAsync(B.fin, state, 18 * nb, cudaMemcpyDeviceToDevice, st));
  VH_CUDA(h, clk.mark(st, &t_fwd));
  if ((r = read_status(h))) return r;

  // ---- observable and seed
  double ndh[2];
  if ((r = eps_p_device<R>(h, state, B.part, B.nd, ndh))) return r;
  if (eps_p) *eps_p = ndh[0] / ndh[1];
  VH_CUDA(h, cudaMemsetAsync(B.xo, 0, NXO3 * nb, st));
  VH_CUDA(h, cudaMemsetAsync(B.xd, 0, 3 * NX3 * nb, st));
  VH_CUDA(h, cudaMemsetAsync(B.yo, 0, NX3 * nb, st));
  VH_CUDA(h, cudaMemsetAsync(B.yd, 0, 3 * NX3 * nb, st));
  VH_CUDA(h, cudaMemsetAsync(B.resb, 0, 9 * nb, st));
  VH_CUDA(h, cudaMemsetAsync(B.dub, 0, 12 * nb, st));
  VH_CUDA(h, cudaMemsetAsync(B.v1tb, 0, 4 * nb, st));
  VH_CUDA(h, cudaMemsetAsync(B.cacc, 0, 2 * n * sizeof(double), st));
  VH_CUDA(h, cudaMemsetAsync(B.ast, 0, sizeof(unsigned), st));
  const long long nint = (long long)C.nx * C.ny * C.nz;
  k_obs3_seed<R><<<grid1(nint, 128), 128, 0, st>>>(C, state, n, B.nd, B.xo);
  VH_CUDA(h, cudaGetLastError());

  Adj3Args<R> a{};
  a.C = C; a.n = n; a.xo = B.xo; a.xd = B.xd; a.yo = B.yo; a.yd = B.yd; a.resb = B.resb; a.dub = B.dub;
  a.v1tb = B.v1tb; a.cacc = B.cacc; a.status = B.ast; a.ts = ts;
  Dir3Args<R> d{};
  d.C = C; d.n = n; d.resb = B.resb; d.dub = B.dub;

  // ---- reverse, one segment at a time
  std::vector<int> seg_marks;
  for (int seg = nseg - 1; seg >= 0; seg--) {
    const int s0 = seg_start(seg), m = (seg + 1 < nseg ? seg_start(seg + 1) : nsteps) - s0;
    int t0, t1, t2;
    VH_CUDA(h, clk.mark(st, &t0));
    if (seg != nseg - 1) {
      VH_CUDA(h, cudaMemcpyAsync(state, B.ck + (size_t)seg * 18 * n, 18 * nb, cudaMemcpyDeviceToDevice, st));
      for (int q = 0; q < m; q++) {
        h->tau = taus[s0 + q];
        if ((r = record_step<R>(h, P, B.Xr + (size_t)q * 18 * n, B.Yr + (size_t)q * kRecY3 * n))) return r;
      }
      VH_CUDA(h, cudaMemcpyAsync(B.Xr + (size_t)m * 18 * n, state, 18 * nb, cudaMemcpyDeviceToDevice, st));
    }
    VH_CUDA(h, clk.mark(st, &t1));
    for (int q = m - 1; q >= 0; q--) {
      const double tau = taus[s0 + q];
      a.X = B.Xr + (size_t)q * 18 * n;
      a.Y = B.Yr + (size_t)q * kRecY3 * n;
      a.X1 = B.Xr + (size_t)(q + 1) * 18 * n;
      a.tau_n = tau;
      k_adj3_stage2<R><<<grid1(nint, 128), 128, 0, st>>>(a);
      d.rec = a.Y; d.kind = REC3_Y; d.tau_s = (R)(tau + ts); d.out = B.yd;
      if ((r = launch_dir3<R>(h, d))) return r;
      k_adj3_stage1<R><<<grid1(nint, 128), 128, 0, st>>>(a);
      d.rec = a.X; d.kind = REC3_X; d.tau_s = (R)tau; d.out = B.xd;
      if ((r = launch_dir3<R>(h, d))) return r;
      VH_CUDA(h, cudaGetLastError());
    }
    VH_CUDA(h, clk.mark(st, &t2));
    seg_marks.push_back(t0);
    seg_marks.push_back(t1);
    seg_marks.push_back(t2);
  }
  if ((r = read_status(h))) return r;

  // ---- gradients of the initial state and of (etas0, etas1)
  k_adj3_final<R><<<grid1(n, 256), 256, 0, st>>>(C, B.ck, n, B.xo, B.xd, grad_state ? B.gs : nullptr,
                                                   grad_e ? B.ge : nullptr);
  sum_cells(B.cacc, n, B.part, B.sums, st);
  VH_CUDA(h, cudaGetLastError());
  double cs[2];
  unsigned astat = 0;
  VH_CUDA(h, cudaMemcpyAsync(cs, B.sums, sizeof(cs), cudaMemcpyDeviceToHost, st));
  VH_CUDA(h, cudaMemcpyAsync(&astat, B.ast, sizeof(astat), cudaMemcpyDeviceToHost, st));
  if (grad_state && (r = pitched_out(h, grad_state, B.gs, 18))) return r;
  if (grad_e && (r = pitched_out(h, grad_e, B.ge, 1))) return r;
  // leave the handle at the final state
  VH_CUDA(h, cudaMemcpyAsync(state, B.fin, 18 * nb, cudaMemcpyDeviceToDevice, st));
  VH_CUDA(h, clk.mark(st, &t_end));
  VH_CUDA(h, cudaStreamSynchronize(st));
  h->tau = taus[nsteps];
  double rec = 0, rev = 0;
  for (size_t k = 0; k + 2 < seg_marks.size(); k += 3) {
    rec += clk.ms(seg_marks[k], seg_marks[k + 1]);
    rev += clk.ms(seg_marks[k + 1], seg_marks[k + 2]);
  }
  h->adj_ms[0] = clk.ms(t_start, t_fwd);
  h->adj_ms[1] = rec;
  h->adj_ms[2] = rev;
  h->adj_ms[3] = clk.ms(t_start, t_end) - h->adj_ms[0] - rec - rev;
  if (grad_etas) { grad_etas[0] = cs[0]; grad_etas[1] = cs[1]; }
  if (astat & AST3_SINGULAR) return fail(h, VH_E_ROOTFIND, "singular root-find Jacobian in the adjoint");
  return VH_OK;
}

}  // namespace

namespace vh {

// the 3+1D discrete adjoint behind vh_adjoint_eps_p (Milne, WENO5, copy
// boundaries; the caller has checked the grid)
int adjoint3_eps_p(vh_handle* h, int nsteps, int every, double* eps_p, double* grad_state, double* grad_e,
                   double* grad_etas) {
  const size_t smem = h->mixed ? dir3_smem<float>(h->C) : dir3_smem<double>(h->C);
  if (smem > 227 * 1024) return fail(h, VH_E_UNSUPPORTED, "vh_adjoint_eps_p: grid line too long for the line kernel");
  return h->mixed ? adjoint3_run<float>(h, h->pf, nsteps, every, eps_p, grad_state, grad_e, grad_etas)
                  : adjoint3_run<double>(h, h->pd, nsteps, every, eps_p, grad_state, grad_e, grad_etas);
}

}  // namespace vh
