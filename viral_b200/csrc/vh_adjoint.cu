// Discrete adjoint of the viscous KT step for boost-invariant Milne grids
// (2+1D, WENO5, copy boundaries; 3+1D grids: vh_adjoint3.cu, dispatched from
// vh_adjoint_eps_p below): gradients of the momentum anisotropy
// eps_p = sum(T^xx - T^yy) / sum(T^xx + T^yy) at the final time with
// respect to the initial state and to the eta/s(T) parameters.
//
// Forward: the ordinary step (step_once), checkpointing the 18 canonical
// fields every k steps.  Reverse, one segment of k steps at a time: restore
// the segment's checkpoint, re-run its steps recording the state at each step
// start (X_n) and after stage 1 (Y_n: e, u, conserved set B), then run the
// reverse of each step, last to first:
//   k_adj_stage2   per interior cell: the ghost images of the cell folded in,
//                  the root of stage 2 by the implicit-function theorem, the
//                  RK2 average, the sources at tau_{n+1} and du/dtau
//   k_adj_dir      one block per x line and per y line: the KT fluxes, WENO
//                  face states and velocity derivatives of stage 2 in reverse
//                  (max-speed and limiter branches are re-taken from the
//                  recorded inputs, so they are the forward pass's)
//   k_adj_stage1   as k_adj_stage2 for stage 1 (sources at tau_n)
//   k_adj_dir      stage 1
// Every adjoint is written by exactly one thread (no atomics), so the
// gradient is deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "vh.h"
#include "vh_adjoint.cuh"
#include "vh_handle.cuh"
#include "vh_adjoint_run.cuh"
#include "vh_nvtx.h"

namespace {

using namespace vh;

// the 10 per-cell inputs of the flux quantities (cell_q), and the three
// prevu adjoints of the own-cell adjoint array (13 fields)
enum : int { XE = 0, XU0 = 1, XP1 = 4, XT0 = 7, XPU0 = 10 };
constexpr int NX = 10, NXO = 13;
// record kinds: X (the 18 canonical fields) and Y (e, u0..u3, B0..B8)
constexpr int REC_X = 0, REC_Y = 1;
constexpr int kRecY = 14;
enum : unsigned { AST_SINGULAR = 1u };

template <class R>
__device__ __forceinline__ void load_cell(const R* rec, int kind, long long n, long long c, R* x) {
  // field offsets of (e, u0, u1, u2, pi^xx, pi^yy, pi^xy, T^tt, T^tx, T^ty)
  if (kind == REC_X) {
    x[0] = rec[c]; x[1] = rec[n + c]; x[2] = rec[2 * n + c]; x[3] = rec[3 * n + c];
    x[4] = rec[5 * n + c]; x[5] = rec[6 * n + c]; x[6] = rec[7 * n + c];
    x[7] = rec[10 * n + c]; x[8] = rec[11 * n + c]; x[9] = rec[12 * n + c];
  } else {
    x[0] = rec[c]; x[1] = rec[n + c]; x[2] = rec[2 * n + c]; x[3] = rec[3 * n + c];
    x[4] = rec[9 * n + c]; x[5] = rec[10 * n + c]; x[6] = rec[11 * n + c];
    x[7] = rec[5 * n + c]; x[8] = rec[6 * n + c]; x[9] = rec[7 * n + c];
  }
}

// WENO velocity derivatives along x and y at an interior cell, as k_dir
// computes them: du9[l*3 + 1 + d] for u^l, l = 0..2 (u0 at U[0])
template <class R>
__device__ __forceinline__ void du_space(const DevCfg& C, const R* U, long long n, long long c, R* du9) {
#pragma unroll
  for (int d = 0; d < 2; d++) {
    const long long s = d == 0 ? 1 : C.px;
    const R h = (R)(d == 0 ? C.dx : C.dy);
#pragma unroll
    for (int l = 0; l < 3; l++) {
      const R* q = U + l * n + c;
      R L, Rr;
      weno_lr<R>(q[-2 * s], q[-s], q[0], q[s], q[2 * s], L, Rr);
      du9[l * 3 + 1 + d] = (L - Rr) / h;
    }
  }
}

// the face ghost cells that the forward fills from interior cell (i, j)
template <class F>
__device__ __forceinline__ void for_images(const DevCfg& C, int i, int j, F&& f) {
  if (i == C.il)
    for (int m = 0; m < NG; m++) f(cix(C, m, j, 0));
  if (i == C.ir - 1)
    for (int m = 0; m < NG; m++) f(cix(C, C.ir + m, j, 0));
  if (j == C.jl)
    for (int m = 0; m < NG; m++) f(cix(C, i, m, 0));
  if (j == C.jr - 1)
    for (int m = 0; m < NG; m++) f(cix(C, i, C.jr + m, 0));
}

template <class R>
struct AdjArgs {
  DevCfg C;
  long long n;
  const R* X;    // record X_n
  const R* Y;    // record Y_n
  const R* X1;   // record X_{n+1}
  R* xo;         // own adjoint of X: 13 fields
  R* xd;         // line adjoints of X: 2 x 10 fields (x lines, y lines)
  R* yo;         // own adjoint of Y: 10 fields
  R* yd;         // line adjoints of Y: 2 x 10 fields
  R* resb;       // 6: adjoint of the flux divergence (T^tt, T^tx, T^ty, pi^xx, pi^yy, pi^xy)
  R* dub;        // 6: adjoint of du^l/dx^d at (l*2 + d)
  R* v1tb;       // 3: adjoint of the stage-1 tau T^{tau mu}
  double* cacc;  // 2 per cell: d/d(etas0, etas1)
  unsigned* status;
  double tau_n, ts;
};

// sum of the own and line adjoints of a recorded state at interior cell c,
// with the adjoints of its ghost images (copies of the cell) folded in
template <class R>
__device__ __forceinline__ void gather_adj(const AdjArgs<R>& a, const R* own, const R* line, int i, int j,
                                           long long c, R* v) {
  const long long n = a.n;
#pragma unroll
  for (int f = 0; f < NX; f++) v[f] = own[f * n + c] + line[f * n + c] + line[(NX + f) * n + c];
  for_images(a.C, i, j, [&](long long g) {
#pragma unroll
    for (int f = 0; f < NX; f++) v[f] += line[f * n + g] + line[(NX + f) * n + g];
  });
}

// adjoint of the root (e, u^x, u^y) -> adjoint of the conserved set it came
// from, added to the direct adjoints v[XT0..], v[XP1..]
template <class R>
__device__ __forceinline__ void root_adjoint(const AdjArgs<R>& a, const R* rec, int kind, long long c, double tau1,
                                             const R* v, R* Tt, R* Pp) {
  const long long n = a.n;
  R x[NX];
  load_cell<R>(rec, kind, n, c, x);
  const double u0 = x[1], u1 = x[2], u2 = x[3];
  const double xb[3] = {(double)v[XE], (double)v[XU0 + 1] + (double)v[XU0] * u1 / u0,
                        (double)v[XU0 + 2] + (double)v[XU0] * u2 / u0};
  const double T3[3] = {x[7], x[8], x[9]}, p3[3] = {x[4], x[5], x[6]}, x3[3] = {x[0], u1, u2};
  double Tb[3] = {0, 0, 0}, pb[3] = {0, 0, 0};
  if (!c2p_ift_vjp(a.C, T3, p3, tau1, x3, xb, Tb, pb)) atomicOr(a.status, AST_SINGULAR);
#pragma unroll
  for (int l = 0; l < 3; l++) {
    Tt[l] = v[XT0 + l] + (R)Tb[l];
    Pp[l] = v[XP1 + l] + (R)pb[l];
  }
}

// Reverse of stage 2 of step n at every interior cell.
template <class R>
__global__ void __launch_bounds__(128) k_adj_stage2(AdjArgs<R> a) {
  const DevCfg& C = a.C;
  const long long n = a.n;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)C.nx * C.ny) return;
  const int i = C.il + (int)(t % C.nx), j = C.jl + (int)(t / C.nx);
  const long long c = cix(C, i, j, 0);
  const double tau1 = a.tau_n + a.ts;
  const R ts = (R)a.ts;

  R v[NX];
  gather_adj<R>(a, a.xo, a.xd, i, j, c, v);
  R pub[3];
#pragma unroll
  for (int l = 0; l < 3; l++) pub[l] = a.xo[(XPU0 + l) * n + c];

  R VT[3], Vp[3];
  root_adjoint<R>(a, a.X1, REC_X, c, tau1, v, VT, Vp);
#pragma unroll
  for (int l = 0; l < 3; l++) VT[l] = VT[l] / (R)tau1;  // A' = Vn / tau1 (T part)

  // Vn = 1/2 tau_n A + 1/2 v1t + 1/2 ts (res + src)   (T^{tau mu})
  //      1/2 A + 1/2 B + 1/2 ts (res + src)           (pi)
  R xn[NXO], yb[NX];
#pragma unroll
  for (int f = 0; f < NXO; f++) xn[f] = 0;
#pragma unroll
  for (int f = 0; f < NX; f++) yb[f] = 0;
  const R half = (R)0.5;
  R rb[6];
#pragma unroll
  for (int l = 0; l < 3; l++) {
    xn[XT0 + l] = half * (R)a.tau_n * VT[l];
    xn[XP1 + l] = half * Vp[l];
    yb[XP1 + l] = half * Vp[l];
    a.v1tb[l * n + c] = half * VT[l];
    rb[l] = half * ts * VT[l];
    rb[3 + l] = half * ts * Vp[l];
  }
  // sources at tau_{n+1} from Y_n; du/dtau = (u(Y) - u(X)) / ts
  const R* Y = a.Y;
  const R ey = Y[c];
  const R uy[3] = {Y[n + c], Y[2 * n + c], Y[3 * n + c]};
  const R py[3] = {Y[9 * n + c], Y[10 * n + c], Y[11 * n + c]};
  R du9[9];
#pragma unroll
  for (int l = 0; l < 3; l++) du9[l * 3] = (uy[l] - a.X[(1 + l) * n + c]) / ts;
  du_space<R>(C, Y + n, n, c, du9);
  const R ob[4] = {rb[0], rb[3], rb[4], rb[5]};
  R eb = 0, ub3[3] = {0, 0, 0}, pb3[3] = {0, 0, 0}, dub9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, cb[2] = {0, 0};
  src2d_vjp<R>(C, (R)tau1, ey, uy, py, du9, ob, eb, ub3, pb3, dub9, cb);
  yb[XE] += eb;
#pragma unroll
  for (int l = 0; l < 3; l++) {
    yb[XU0 + l] += ub3[l] + dub9[l * 3] / ts;
    yb[XP1 + l] += pb3[l];
    xn[XU0 + l] += pub[l] - dub9[l * 3] / ts;  // prevu of X_{n+1} is u of X_n
  }
#pragma unroll
  for (int f = 0; f < NXO; f++) a.xo[f * n + c] = xn[f];
#pragma unroll
  for (int f = 0; f < NX; f++) a.yo[f * n + c] = yb[f];
#pragma unroll
  for (int q = 0; q < 6; q++) a.resb[q * n + c] = rb[q];
#pragma unroll
  for (int l = 0; l < 3; l++) {
    a.dub[(l * 2) * n + c] = dub9[l * 3 + 1];
    a.dub[(l * 2 + 1) * n + c] = dub9[l * 3 + 2];
  }
  a.cacc[c] += (double)cb[0];
  a.cacc[n + c] += (double)cb[1];
}

// Reverse of stage 1 of step n at every interior cell.
template <class R>
__global__ void __launch_bounds__(128) k_adj_stage1(AdjArgs<R> a) {
  const DevCfg& C = a.C;
  const long long n = a.n;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)C.nx * C.ny) return;
  const int i = C.il + (int)(t % C.nx), j = C.jl + (int)(t / C.nx);
  const long long c = cix(C, i, j, 0);
  const double tau1 = a.tau_n + a.ts;
  const R ts = (R)a.ts;

  R w[NX];
  gather_adj<R>(a, a.yo, a.yd, i, j, c, w);
  R VT[3], Vp[3];
  root_adjoint<R>(a, a.Y, REC_Y, c, tau1, w, VT, Vp);
#pragma unroll
  for (int l = 0; l < 3; l++) VT[l] = VT[l] / (R)tau1 + a.v1tb[l * n + c];  // B = Vn / tau1, v1t = Vn

  // Vn = tau_n A + ts (res + src)   (T^{tau mu});   A + ts (res + src)   (pi)
  R xn[NXO];
#pragma unroll
  for (int f = 0; f < NXO; f++) xn[f] = a.xo[f * n + c];
  R rb[6];
#pragma unroll
  for (int l = 0; l < 3; l++) {
    xn[XT0 + l] += (R)a.tau_n * VT[l];
    xn[XP1 + l] += Vp[l];
    rb[l] = ts * VT[l];
    rb[3 + l] = ts * Vp[l];
  }
  const R* X = a.X;
  const R ex = X[c];
  const R ux[3] = {X[n + c], X[2 * n + c], X[3 * n + c]};
  const R px[3] = {X[5 * n + c], X[6 * n + c], X[7 * n + c]};
  R du9[9];
#pragma unroll
  for (int l = 0; l < 3; l++) du9[l * 3] = (ux[l] - X[(14 + l) * n + c]) / ts;
  du_space<R>(C, X + n, n, c, du9);
  const R ob[4] = {rb[0], rb[3], rb[4], rb[5]};
  R eb = 0, ub3[3] = {0, 0, 0}, pb3[3] = {0, 0, 0}, dub9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, cb[2] = {0, 0};
  src2d_vjp<R>(C, (R)a.tau_n, ex, ux, px, du9, ob, eb, ub3, pb3, dub9, cb);
  xn[XE] += eb;
#pragma unroll
  for (int l = 0; l < 3; l++) {
    xn[XU0 + l] += ub3[l] + dub9[l * 3] / ts;
    xn[XPU0 + l] -= dub9[l * 3] / ts;
    xn[XP1 + l] += pb3[l];
  }
#pragma unroll
  for (int f = 0; f < NXO; f++) a.xo[f * n + c] = xn[f];
#pragma unroll
  for (int q = 0; q < 6; q++) a.resb[q * n + c] = rb[q];
#pragma unroll
  for (int l = 0; l < 3; l++) {
    a.dub[(l * 2) * n + c] = dub9[l * 3 + 1];
    a.dub[(l * 2 + 1) * n + c] = dub9[l * 3 + 2];
  }
  a.cacc[c] += (double)cb[0];
  a.cacc[n + c] += (double)cb[1];
}

template <class R>
struct DirArgs {
  DevCfg C;
  long long n;
  const R* rec;  // recorded primal state of the stage
  int kind;      // REC_X or REC_Y
  R tau_s;       // time the stage's fluxes were formed at
  const R* resb;
  const R* dub;
  R* out;        // 2 x 10 fields: line adjoints (x lines, then y lines)
};

// quantities whose WENO stencils are reversed at the same time, threads per
// line block, and shared-memory words per line cell
constexpr int kQP = 4;
constexpr int kDirWords = 55 + 5 * kQP;
// threads per line block: two blocks per SM keep all the lines of a 128^2
// grid (256 blocks) resident in one wave at either precision
template <class R>
struct DirShape {
  static constexpr int threads = sizeof(R) == 8 ? 256 : 512;
};

template <class R>
__device__ __forceinline__ R sgn(R x) { return (R)((x > (R)0) - (x < (R)0)); }

// Reverse of the flux sweep of one stage along one line.  The whole line
// (interior and both ghost layers) sits in shared memory, so the scatter of
// the WENO stencils stays inside the block; each cell's line adjoint is
// written once.
template <class R, int DIR>
__device__ __forceinline__ void adj_line(const DirArgs<R>& a, int line, R* sm) {
  const DevCfg& C = a.C;
  const long long n = a.n;
  const int G = DIR == 0 ? C.gx : C.gy;
  const int lo = DIR == 0 ? C.il : C.jl, hi = DIR == 0 ? C.ir : C.jr;
  const long long stride = DIR == 0 ? 1 : C.px;
  const long long base = DIR == 0 ? cix(C, 0, C.jl + line, 0) : cix(C, C.il + line, 0, 0);
  const double hh = DIR == 0 ? C.dx : C.dy;
  const R h = (R)hh, inv_h = (R)(1.0 / hh);
  R* q = sm;            // 13: flux quantities
  R* lv = q + 13 * G;   // 7: face state at the right face (V^0..5, speed)
  R* rv = lv + 7 * G;   // 7: face state at the left face
  R* hb = rv + 7 * G;   // 6: adjoint of the KT flux at the face right of cell f
  R* am = hb + 6 * G;   // max signal speed at that face
  R* sl = am + G;       // adjoint of the speed's right-face state
  R* sr = sl + G;       // adjoint of the speed's left-face state
  R* qb = sr + G;       // 16: adjoints of the 13 quantities and of u^0..2
  R* uu = qb + 16 * G;  // 3: u^0..2 along the line
  R* c5 = uu + 3 * G;   // 5 x kQP: stencil contributions of the quantities in flight
  const int tid = threadIdx.x, nt = blockDim.x;

  for (int i = tid; i < G; i += nt) {
    R x[NX], ql[NQ];
    load_cell<R>(a.rec, a.kind, n, base + i * stride, x);
    cell_q<R, DIR>(C, a.tau_s, x, i >= lo && i < hi, ql);
#pragma unroll
    for (int k = 0; k < NQ; k++) q[k * G + i] = ql[k];
#pragma unroll
    for (int l = 0; l < 3; l++) uu[l * G + i] = x[1 + l];
#pragma unroll
    for (int k = 0; k < 16; k++) qb[k * G + i] = 0;
    sl[i] = 0;
    sr[i] = 0;
  }
  __syncthreads();
  const int ns = hi - lo + 2;  // cells lo-1 .. hi have full stencils
  for (int w = tid; w < 7 * ns; w += nt) {
    const int k = w / ns, i = lo - 1 + w % ns;
    const R* s = q + (6 + k) * G + i;
    weno_lr<R>(s[-2], s[-1], s[0], s[1], s[2], lv[k * G + i], rv[k * G + i]);
  }
  __syncthreads();
  // faces f | f+1 for f in [lo-1, hi-1]
  for (int f = lo - 1 + tid; f <= hi - 1; f += nt) {
    const long long cf = base + f * stride, cn = cf + stride;
    const R L = lv[6 * G + f], Rn = rv[6 * G + f + 1];
    const bool diss = f + 1 != lo;  // no dissipation left of the first interior cell
    const R amax = diss ? fmax(fabs(L), fabs(Rn)) : (R)0;
    R amb = 0;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const R rf = f >= lo ? a.resb[k * n + cf] : (R)0;
      const R rn = f + 1 < hi ? a.resb[k * n + cn] : (R)0;
      const R H = (rn - rf) * inv_h;  // res_i = -(H_{i+1/2} - H_{i-1/2}) / h
      hb[k * G + f] = H;
      amb -= (R)0.5 * (rv[k * G + f + 1] - lv[k * G + f]) * H;
    }
    am[f] = amax;
    if (diss) {
      if (fabs(L) >= fabs(Rn)) sl[f] = amb * sgn(L);
      else sr[f + 1] = amb * sgn(Rn);
    }
  }
  __syncthreads();
  // WENO stencils in reverse, kQP quantities at a time (the 13 flux
  // quantities, then the three velocity lines of the derivative du^l/dx)
  for (int k0 = 0; k0 < 16; k0 += kQP) {
    for (int w = tid; w < kQP * G; w += nt) {
      const int kq = w / G, i = w % G, k = k0 + kq;
      R cc[5] = {0, 0, 0, 0, 0};
      if (k < 16 && i >= lo - 1 && i <= hi) {
        const bool hasL = i <= hi - 1, hasR = i >= lo;  // faces i and i-1
        R Lb = 0, Rb = 0;
        if (k < 6) {
          if (hasL) Lb = (R)0.5 * hb[k * G + i];
          if (hasR) Rb = (R)0.5 * hb[k * G + i - 1];
        } else if (k < 12) {
          if (hasL) Lb = (R)0.5 * am[i] * hb[(k - 6) * G + i];
          if (hasR) Rb = -(R)0.5 * am[i - 1] * hb[(k - 6) * G + i - 1];
        } else if (k == 12) {
          Lb = sl[i];
          Rb = sr[i];
        } else if (i >= lo && i < hi) {
          const R d = a.dub[((k - 13) * 2 + DIR) * n + base + i * stride];
          Lb = d / h;
          Rb = -d / h;
        }
        const R* s = k < 13 ? q + k * G : uu + (k - 13) * G;
        if (Lb != (R)0 || Rb != (R)0) weno_lr_vjp<R>(s + i - 2, Lb, Rb, cc);
      }
#pragma unroll
      for (int o = 0; o < 5; o++) c5[(kq * 5 + o) * G + i] = cc[o];
    }
    __syncthreads();
    for (int w = tid; w < kQP * G; w += nt) {
      const int kq = w / G, jj = w % G, k = k0 + kq;
      R acc = 0;
#pragma unroll
      for (int o = 0; o < 5; o++) {
        const int i = jj + 2 - o;
        if (i >= 0 && i < G) acc += c5[(kq * 5 + o) * G + i];
      }
      if (k < 16) qb[k * G + jj] += acc;
    }
    __syncthreads();
  }
  for (int jj = tid; jj < G; jj += nt) {
    const long long c = base + jj * stride;
    R x[NX], qbl[NQ], xb[NX];
    load_cell<R>(a.rec, a.kind, n, c, x);
#pragma unroll
    for (int k = 0; k < NQ; k++) qbl[k] = qb[k * G + jj];
#pragma unroll
    for (int f = 0; f < NX; f++) xb[f] = 0;
    cell_q_vjp<R, DIR>(C, a.tau_s, x, jj >= lo && jj < hi, qbl, xb);
#pragma unroll
    for (int l = 0; l < 3; l++) xb[1 + l] += qb[(13 + l) * G + jj];
    R* out = a.out + (long long)DIR * NX * n;
#pragma unroll
    for (int f = 0; f < NX; f++) out[f * n + c] = xb[f];
  }
}

// blockIdx.y = direction, blockIdx.x = line
template <class R>
__global__ void __launch_bounds__(DirShape<R>::threads, 2) k_adj_dir(DirArgs<R> a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  R* sm = reinterpret_cast<R*>(smem_raw);
  if (blockIdx.y == 0) {
    if ((int)blockIdx.x < a.C.ny) adj_line<R, 0>(a, blockIdx.x, sm);
  } else {
    if ((int)blockIdx.x < a.C.nx) adj_line<R, 1>(a, blockIdx.x, sm);
  }
}

// adjoint seed: d eps_p / d (e, u^x, u^y, pi^xx, pi^yy) of the final state
template <class R>
__global__ void k_obs_seed(DevCfg C, const R* S, long long n, const double* nd, R* xo) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)C.nx * C.ny) return;
  const int i = C.il + (int)(t % C.nx), j = C.jl + (int)(t / C.nx);
  const long long c = cix(C, i, j, 0);
  R eb, u1b, u2b, p1b, p2b;
  obs_cell_vjp<R>(C, S[c], S[2 * n + c], S[3 * n + c], nd[0], nd[1], eb, u1b, u2b, p1b, p2b);
  xo[XE * n + c] = eb;
  xo[(XU0 + 1) * n + c] = u1b;
  xo[(XU0 + 2) * n + c] = u2b;
  xo[XP1 * n + c] = p1b;
  xo[(XP1 + 1) * n + c] = p2b;
}

// gradients of the initial state: the 18 canonical fields (every field an
// independent variable) and the energy density of vh_init_profile (T^{tau mu}
// re-derived from e at fixed u and pi)
template <class R>
__global__ void k_adj_final(DevCfg C, const R* X0, long long n, const R* xo, const R* xd, double* gs, double* ge) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  double v[NX];
  for (int f = 0; f < NX; f++) v[f] = (double)xo[f * n + c] + (double)xd[f * n + c] + (double)xd[(NX + f) * n + c];
  if (gs) {
    for (int f = 0; f < 18; f++) gs[f * n + c] = 0.0;
    gs[c] = v[XE];
    for (int l = 0; l < 3; l++) {
      gs[(1 + l) * n + c] = v[XU0 + l];
      gs[(5 + l) * n + c] = v[XP1 + l];
      gs[(10 + l) * n + c] = v[XT0 + l];
      gs[(14 + l) * n + c] = (double)xo[(XPU0 + l) * n + c];
    }
  }
  if (ge) {
    double P, dP, T, dT;
    eos_d<double>(C, (double)X0[c], P, dP, T, dT);
    const double u0 = X0[n + c], u1 = X0[2 * n + c], u2 = X0[3 * n + c];
    ge[c] = v[XE] + v[XT0] * ((1 + dP) * u0 * u0 - dP) + v[XT0 + 1] * (1 + dP) * u0 * u1 +
            v[XT0 + 2] * (1 + dP) * u0 * u2;
  }
}

template <class R>
size_t dir_smem(const DevCfg& C) {
  return (size_t)kDirWords * std::max(C.gx, C.gy) * sizeof(R);
}

template <class R>
int adjoint_run(vh_handle* h, const DevPtrs<R>& P, int nsteps, int every, double* eps_p, double* grad_state,
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
  const int last0 = seg_start(nseg - 1);  // first step of the last segment

  // ---- workspace
  Carve cv;
  auto layout = [&](Carve& c, R** ck, R** fin, R** Xr, R** Yr, R** xo, R** xd, R** yo, R** yd, R** resb, R** dub,
                    R** v1tb, double** cacc, double** part, double** nd, double** sums, unsigned** ast, double** gs,
                    double** ge) {
    *ck = c.take<R>((size_t)nseg * 18 * n);
    *fin = c.take<R>((size_t)18 * n);
    *Xr = c.take<R>((size_t)(seg_len + 1) * 18 * n);
    *Yr = c.take<R>((size_t)seg_len * kRecY * n);
    *xo = c.take<R>((size_t)NXO * n);
    *xd = c.take<R>((size_t)2 * NX * n);
    *yo = c.take<R>((size_t)NX * n);
    *yd = c.take<R>((size_t)2 * NX * n);
    *resb = c.take<R>((size_t)6 * n);
    *dub = c.take<R>((size_t)6 * n);
    *v1tb = c.take<R>((size_t)3 * n);
    *cacc = c.take<double>((size_t)2 * n);
    *part = c.take<double>((size_t)2 * kObsBlocks);
    *nd = c.take<double>(2);
    *sums = c.take<double>(2);
    *ast = c.take<unsigned>(1);
    *gs = c.take<double>((size_t)18 * n);
    *ge = c.take<double>((size_t)n);
  };
  R *ck, *fin, *Xr, *Yr, *xo, *xd, *yo, *yd, *resb, *dub, *v1tb;
  double *cacc, *part, *nd, *sums, *gs_dev, *ge_dev;
  unsigned* ast;
  layout(cv, &ck, &fin, &Xr, &Yr, &xo, &xd, &yo, &yd, &resb, &dub, &v1tb, &cacc, &part, &nd, &sums, &ast, &gs_dev,
         &ge_dev);
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
  layout(cw, &ck, &fin, &Xr, &Yr, &xo, &xd, &yo, &yd, &resb, &dub, &v1tb, &cacc, &part, &nd, &sums, &ast, &gs_dev,
         &ge_dev);
  const size_t smem = dir_smem<R>(C);
  VH_CUDA(h, cudaFuncSetAttribute(k_adj_dir<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
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
      VH_CUDA(h, cudaMemcpyAsync(ck + (size_t)k * 18 * n, state, 18 * nb, cudaMemcpyDeviceToDevice, st));
    }
    taus[s] = h->tau;
    if (s >= last0) r = record_step<R>(h, P, Xr + (size_t)(s - last0) * 18 * n, Yr + (size_t)(s - last0) * kRecY * n);
    else r = step_once<R>(h, P);
    if (r) return r;
  }
  taus[nsteps] = h->tau;
  VH_CUDA(h, cudaMemcpyAsync(Xr + (size_t)(nsteps - last0) * 18 * n, state, 18 * nb, cudaMemcpyDeviceToDevice, st));
  VH_CUDA(h, cudaMemcpyAsync(fin, state, 18 * nb, cudaMemcpyDeviceToDevice, st));
  VH_CUDA(h, clk.mark(st, &t_fwd));
  if ((r = read_status(h))) return r;

  // ---- observable and seed
  double ndh[2];
  if ((r = eps_p_device<R>(h, state, part, nd, ndh))) return r;
  if (eps_p) *eps_p = ndh[0] / ndh[1];
  VH_CUDA(h, cudaMemsetAsync(xo, 0, NXO * nb, st));
  VH_CUDA(h, cudaMemsetAsync(xd, 0, 2 * NX * nb, st));
  VH_CUDA(h, cudaMemsetAsync(yo, 0, NX * nb, st));
  VH_CUDA(h, cudaMemsetAsync(yd, 0, 2 * NX * nb, st));
  VH_CUDA(h, cudaMemsetAsync(resb, 0, 6 * nb, st));
  VH_CUDA(h, cudaMemsetAsync(dub, 0, 6 * nb, st));
  VH_CUDA(h, cudaMemsetAsync(v1tb, 0, 3 * nb, st));
  VH_CUDA(h, cudaMemsetAsync(cacc, 0, 2 * n * sizeof(double), st));
  VH_CUDA(h, cudaMemsetAsync(ast, 0, sizeof(unsigned), st));
  const long long nint = (long long)C.nx * C.ny;
  k_obs_seed<R><<<grid1(nint, 128), 128, 0, st>>>(C, state, n, nd, xo);
  VH_CUDA(h, cudaGetLastError());

  AdjArgs<R> a{};
  a.C = C; a.n = n; a.xo = xo; a.xd = xd; a.yo = yo; a.yd = yd; a.resb = resb; a.dub = dub; a.v1tb = v1tb;
  a.cacc = cacc; a.status = ast; a.ts = ts;
  DirArgs<R> d{};
  d.C = C; d.n = n; d.resb = resb; d.dub = dub;
  const int G = std::max(C.gx, C.gy);
  const int dthreads = DirShape<R>::threads;
  const dim3 dgrid(std::max(C.nx, C.ny), 2);

  // ---- reverse, one segment at a time
  std::vector<int> seg_marks;
  for (int seg = nseg - 1; seg >= 0; seg--) {
    const int s0 = seg_start(seg), m = (seg + 1 < nseg ? seg_start(seg + 1) : nsteps) - s0;
    int t0, t1, t2;
    VH_CUDA(h, clk.mark(st, &t0));
    if (seg != nseg - 1) {
      VH_CUDA(h, cudaMemcpyAsync(state, ck + (size_t)seg * 18 * n, 18 * nb, cudaMemcpyDeviceToDevice, st));
      for (int q = 0; q < m; q++) {
        h->tau = taus[s0 + q];
        if ((r = record_step<R>(h, P, Xr + (size_t)q * 18 * n, Yr + (size_t)q * kRecY * n))) return r;
      }
      VH_CUDA(h, cudaMemcpyAsync(Xr + (size_t)m * 18 * n, state, 18 * nb, cudaMemcpyDeviceToDevice, st));
    }
    VH_CUDA(h, clk.mark(st, &t1));
    for (int q = m - 1; q >= 0; q--) {
      const double tau = taus[s0 + q];
      a.X = Xr + (size_t)q * 18 * n;
      a.Y = Yr + (size_t)q * kRecY * n;
      a.X1 = Xr + (size_t)(q + 1) * 18 * n;
      a.tau_n = tau;
      k_adj_stage2<R><<<grid1(nint, 128), 128, 0, st>>>(a);
      d.rec = a.Y; d.kind = REC_Y; d.tau_s = (R)(tau + ts); d.out = yd;
      k_adj_dir<R><<<dgrid, dthreads, smem, st>>>(d);
      k_adj_stage1<R><<<grid1(nint, 128), 128, 0, st>>>(a);
      d.rec = a.X; d.kind = REC_X; d.tau_s = (R)tau; d.out = xd;
      k_adj_dir<R><<<dgrid, dthreads, smem, st>>>(d);
      VH_CUDA(h, cudaGetLastError());
    }
    VH_CUDA(h, clk.mark(st, &t2));
    seg_marks.push_back(t0);
    seg_marks.push_back(t1);
    seg_marks.push_back(t2);
  }
  if ((r = read_status(h))) return r;

  // ---- gradients of the initial state and of (etas0, etas1)
  k_adj_final<R><<<grid1(n, 256), 256, 0, st>>>(C, ck, n, xo, xd, grad_state ? gs_dev : nullptr,
                                                  grad_e ? ge_dev : nullptr);
  sum_cells(cacc, n, part, sums, st);
  VH_CUDA(h, cudaGetLastError());
  double cs[2];
  unsigned astat = 0;
  VH_CUDA(h, cudaMemcpyAsync(cs, sums, sizeof(cs), cudaMemcpyDeviceToHost, st));
  VH_CUDA(h, cudaMemcpyAsync(&astat, ast, sizeof(astat), cudaMemcpyDeviceToHost, st));
  if (grad_state && (r = pitched_out(h, grad_state, gs_dev, 18))) return r;
  if (grad_e && (r = pitched_out(h, grad_e, ge_dev, 1))) return r;
  // leave the handle at the final state
  VH_CUDA(h, cudaMemcpyAsync(state, fin, 18 * nb, cudaMemcpyDeviceToDevice, st));
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
  if (astat & AST_SINGULAR) return fail(h, VH_E_ROOTFIND, "singular root-find Jacobian in the adjoint");
  return VH_OK;
}

}  // namespace

extern "C" int vh_eps_p(vh_handle* h, double* eps_p) {
  if (!h || !eps_p) return VH_E_ARG;
  if (!h->have_state) return fail(h, VH_E_STATE, "no state set");
  if (h->C.cart) return fail(h, VH_E_UNSUPPORTED, "vh_eps_p: Milne grids only");
  double* buf = nullptr;
  VH_CUDA(h, cudaMallocAsync(&buf, sizeof(double) * (2 * kObsBlocks + 2), h->stream));
  double nd[2];
  const int r = h->mixed ? eps_p_device<float>(h, static_cast<const float*>(h->state), buf, buf + 2 * kObsBlocks, nd)
                         : eps_p_device<double>(h, static_cast<const double*>(h->state), buf, buf + 2 * kObsBlocks, nd);
  cudaFreeAsync(buf, h->stream);
  if (r) return r;
  *eps_p = nd[0] / nd[1];
  return VH_OK;
}

extern "C" int vh_adjoint_phase_times(const vh_handle* h, double* ms4) {
  if (!h || !ms4) return VH_E_ARG;
  for (int q = 0; q < 4; q++) ms4[q] = h->adj_ms[q];
  return VH_OK;
}

extern "C" int vh_adjoint_eps_p(vh_handle* h, int nsteps, int checkpoint_every, double* eps_p, double* grad_state,
                                double* grad_e, double* grad_etas) {
  if (!h || nsteps < 1 || checkpoint_every < 1) return VH_E_ARG;
  if (!h->have_state) return fail(h, VH_E_STATE, "no state set");
  VhNvtxRange range("discrete adjoint of eps_p");
  const DevCfg& C = h->C;
  if (C.cart || C.mirror || C.recon != VH_RECON_WENO5 || C.cold)
    return fail(h, VH_E_UNSUPPORTED,
                "vh_adjoint_eps_p: Milne grids with WENO reconstruction and copy boundaries only");
  if (!C.bi) return adjoint3_eps_p(h, nsteps, checkpoint_every, eps_p, grad_state, grad_e, grad_etas);
  const size_t smem = h->mixed ? dir_smem<float>(C) : dir_smem<double>(C);
  if (smem > 227 * 1024)
    return fail(h, VH_E_UNSUPPORTED, "vh_adjoint_eps_p: grid line too long for the line kernel");
  return h->mixed ? adjoint_run<float>(h, h->pf, nsteps, checkpoint_every, eps_p, grad_state, grad_e, grad_etas)
                  : adjoint_run<double>(h, h->pd, nsteps, checkpoint_every, eps_p, grad_state, grad_e, grad_etas);
}
