// Kernels of one RK stage of the viscous KT step and its helpers.
//
// A stage is D+1 launches (D = 2 or 3 directions):
//   k_dir<DIR>  one per direction (k_dir_tma when the tile arrives by TMA
//               box copies): stages a tile of cells plus 3 halo cells along
//               DIR in shared memory as (F^DIR, tau T^{tau mu}, pi, speed),
//               forms WENO5 (or minmod) face states and the KT flux at every
//               face of the tile, adds the flux difference to the divergence
//               accumulator, and writes the WENO velocity derivative along
//               DIR (NEWEST5/hydroKT.h:16-491, NEWEST5/Source.h:3-101).
//   k_update    one thread per interior cell: sources, RK2 combination,
//               FP64 root-find, and the ghost copy of boundary cells
//               (NEWEST5/Source.h:165-433, time.h:1-387, multiroot.h:331-493,
//               boundary.h:1-276).
#pragma once

#include <cuda.h>

#include "vh_device.cuh"

namespace vh {

// Tile shapes: NA = 32 cells along the direction (6 of them halo, so 26
// outputs), NC lines across it.  Loads run x-fastest (coalesced); in the
// compute phase each warp owns one line and its lanes walk along it.
template <int DIR, class R>
struct Tile;
template <class R>
struct Tile<0, R> { static constexpr int NA = 32, NC = 4; };
template <class R>
struct Tile<1, R> { static constexpr int NA = 32, NC = 8; };
template <class R>
struct Tile<2, R> { static constexpr int NA = 32, NC = 8; };

template <class R, int DIR, int NC_ = Tile<DIR, R>::NC>
struct DirSmem {
  static constexpr int NA = Tile<DIR, R>::NA, NC = NC_;
  static constexpr int TL = NA - 6;
  static constexpr int LD = NA + 1;  // padded line length (bank spread)
  // F^l and Var^l of a cell side by side, and the velocity as the pairs
  // (u^tau, u^x), (u^y, u^eta): the reconstruction takes both members of a
  // pair with one shared-memory load (8 bytes in FP32, 16 in FP64)
  alignas(16) R fv[9][NC * LD][2];
  R spd[NC * LD];                   // signal speed
  alignas(16) R up[2][NC * LD][2];  // u^mu for the velocity derivative
};

// both members of a pair at line position s
__device__ __forceinline__ unsigned long long ld_pair(const float (*a)[2], int s) {
  return *reinterpret_cast<const unsigned long long*>(a[s]);
}
__device__ __forceinline__ double2 ld_pair(const double (*a)[2], int s) {
  return *reinterpret_cast<const double2*>(a[s]);
}

// Centre flux along DIR, Var and signal speed of one cell
// (NEWEST5/hydroKT.h:16-83, 161-245, 349-367).
template <class R, int DIR>
__device__ inline void cell_terms(const DevCfg& C, R tau, R e, const R* u, const R* p, const R* T, bool interior,
                                  R* F, R* V, R& spd) {
  const bool cart = C.cart;
  const R t2 = cart ? (R)1 : tau * tau;
  const R tf = cart ? (R)1 : tau;
  const R P = eos_P<R>(C, e);
  const R ep = e + P;
  const R u0 = u[0], u1 = u[1], u2 = u[2], u3 = u[3];
  PiDep<R> d = pi_dep<R>(u0, u1, u2, u3, p, t2);
  const R iu0 = (R)1 / u0;
  if (DIR == 0) {
    F[0] = tf * (d.tx + u1 * u0 * ep);
    F[1] = tf * (p[0] + P + u1 * u1 * ep);
    F[2] = tf * (p[2] + u1 * u2 * ep);
    F[3] = tf * (p[3] + u1 * u3 * ep);
#pragma unroll
    for (int l = 0; l < 5; l++) F[4 + l] = (p[l] * u1) * iu0;
    spd = interior ? u1 * iu0 : (R)0;
  } else if (DIR == 1) {
    F[0] = tf * (d.ty + u2 * u0 * ep);
    F[1] = tf * (p[2] + u2 * u1 * ep);
    F[2] = tf * (p[1] + P + u2 * u2 * ep);
    F[3] = tf * (p[4] + u2 * u3 * ep);
#pragma unroll
    for (int l = 0; l < 5; l++) F[4 + l] = (p[l] * u2) * iu0;
    spd = interior ? u2 * iu0 : (R)0;
  } else {
    F[0] = tf * (d.te + u3 * u0 * ep);
    F[1] = tf * (p[3] + u3 * u1 * ep);
    F[2] = tf * (p[4] + u3 * u2 * ep);
    F[3] = cart ? (d.ee + P + u3 * u3 * ep) : tf * (d.ee + P / t2 + u3 * u3 * ep);
    // the eta flux of pi carries a factor tau (NEWEST5/hydroKT.h:76-81)
#pragma unroll
    for (int l = 0; l < 5; l++) F[4 + l] = cart ? (p[l] * u3) * iu0 : tau * (p[l] * u3) * iu0;
    spd = interior ? (cart ? u3 * iu0 : tau * u3 * iu0) : (R)0;
  }
#pragma unroll
  for (int l = 0; l < 4; l++) V[l] = cart ? T[l] : tf * T[l];
#pragma unroll
  for (int l = 0; l < 5; l++) V[4 + l] = p[l];
}

// Both face states of the stencil centred on the lane's cell: L at the
// right face, R at the left face (WENO5, or generalized minmod).  Line
// position k of the quantity is q[k * ST].
template <class R, int ST = 1>
__device__ inline void recon_lr(const DevCfg& C, const R* q, int s, R& L, R& Rr) {
  if (C.recon == 0) {
    weno_lr<R>(q[(s - 2) * ST], q[(s - 1) * ST], q[s * ST], q[(s + 1) * ST], q[(s + 2) * ST], L, Rr);
  } else {
    L = mm_left<R>((R)C.mm_theta, q[(s - 1) * ST], q[s * ST], q[(s + 1) * ST]);
    Rr = mm_right<R>((R)C.mm_theta, q[(s - 1) * ST], q[s * ST], q[(s + 1) * ST]);
  }
}

// Paired FP32 arithmetic (sm_100's f32x2 add/mul/fma: one instruction for
// two lanes of a 64-bit register pair).  The FP32 sweeps reconstruct the
// flux F^l and the conserved variable V^l of a face together, so the WENO5
// arithmetic of the pair runs at half the instruction count; each lane
// rounds as the scalar operation would.
struct F2 {
  unsigned long long v;
};
__device__ __forceinline__ F2 f2(float a, float b) {
  F2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ F2 f2s(float a) { return f2(a, a); }
__device__ __forceinline__ void f2u(F2 x, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(x.v));
}
__device__ __forceinline__ F2 add2(F2 a, F2 b) {
  F2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 sub2(F2 a, F2 b) {
  F2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 mul2(F2 a, F2 b) {
  F2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) {
  F2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}

// weno_lr for two quantities at once (same formulas as weno_beta/weno_lr)
__device__ __forceinline__ void weno_lr2(F2 qm2, F2 qm1, F2 qc, F2 qp1, F2 qp2, F2& L, F2& Rr) {
  const F2 c13 = f2s((float)(13. / 12.)), q4 = f2s(0.25f), two = f2s(2.f), m2 = f2s(-2.f), three = f2s(3.f),
           m4 = f2s(-4.f), five = f2s(5.f), m7 = f2s(-7.f), eleven = f2s(11.f), eps = f2s(1e-6f);
  F2 a = add2(fma2(m2, qp1, qc), qp2), c = add2(fma2(m4, qp1, mul2(three, qc)), qp2);
  const F2 b0 = fma2(c13, mul2(a, a), mul2(q4, mul2(c, c)));
  a = add2(fma2(m2, qc, qm1), qp1);
  c = sub2(qm1, qp1);
  const F2 b1 = fma2(c13, mul2(a, a), mul2(q4, mul2(c, c)));
  a = add2(fma2(m2, qm1, qm2), qc);
  c = fma2(three, qc, fma2(m4, qm1, qm2));
  const F2 b2 = fma2(c13, mul2(a, a), mul2(q4, mul2(c, c)));
  const F2 e0 = add2(eps, b0), e1 = add2(eps, b1), e2 = add2(eps, b2);
  const F2 E0 = mul2(e0, e0), E1 = mul2(e1, e1), E2 = mul2(e2, e2);
  const F2 P12 = mul2(E1, E2), P02 = mul2(E0, E2), P01 = mul2(E0, E1);
  const F2 nl0 = mul2(f2s(0.3f), P12), nl1 = mul2(f2s(0.6f), P02), nl2 = mul2(f2s(0.1f), P01);
  const F2 nr0 = mul2(f2s(0.1f), P12), nr2 = mul2(f2s(0.3f), P01);
  const F2 ql0 = sub2(fma2(five, qp1, mul2(two, qc)), qp2);
  const F2 ql1 = fma2(two, qp1, fma2(five, qc, sub2(f2s(0.f), qm1)));
  const F2 ql2 = fma2(eleven, qc, fma2(m7, qm1, mul2(two, qm2)));
  const F2 qr0 = fma2(two, qp2, fma2(m7, qp1, mul2(eleven, qc)));
  const F2 qr1 = sub2(fma2(five, qc, mul2(two, qm1)), qp1);
  const F2 qr2 = fma2(two, qc, fma2(five, qm1, sub2(f2s(0.f), qm2)));
  const F2 numl = fma2(nl2, ql2, fma2(nl1, ql1, mul2(nl0, ql0)));
  const F2 numr = fma2(nr2, qr2, fma2(nl1, qr1, mul2(nr0, qr0)));
  const F2 six = f2s(6.f);
  const F2 denl = mul2(six, add2(add2(nl0, nl1), nl2)), denr = mul2(six, add2(add2(nr0, nl1), nr2));
  float a0, a1, d0, d1;
  f2u(numl, a0, a1);
  f2u(denl, d0, d1);
  L = f2(__fdividef(a0, d0), __fdividef(a1, d1));
  f2u(numr, a0, a1);
  f2u(denr, d0, d1);
  Rr = f2(__fdividef(a0, d0), __fdividef(a1, d1));
}

// Programmatic dependent launch: the step's kernels are launched so that the
// next one may start while this one's last blocks still run.  Every block
// first waits until the previous kernel in the stream has completed and its
// writes are visible (a no-op under an ordinary launch), then lets the next
// kernel be launched.
__device__ __forceinline__ void pdl_wait_then_release() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ---- TMA staging of a sweep's tile (cp.async.bulk.tensor, one mbarrier)
//
// The state is one 4D tensor (x over the padded row pitch, y, z, array):
// the 52 arrays back to back.  A tile of the sweep along DIR is two box
// copies: arrays 0..4 (e, u^mu) and the nine arrays of the conserved set it
// reads (set A: pi 5..9 then T^{tau mu} 10..13; set B: T^{tau mu} 18..21
// then pi 22..26).  Along x the box's start is rounded down to a 16-byte
// boundary (4 floats, 2 doubles) and the box is wide enough for the tile
// from there; across x (the y and eta sweeps) the tile starts on a multiple
// of NC cells of the padded row, so the box is exactly the tile's NC lines.
// Cells outside the tensor are filled with zeros by the copy and, like the
// cells outside the grid, never used.
template <class R, int DIR, int NC>
struct TmaBox {
  static constexpr int XA = sizeof(R) == 4 ? 4 : 2;  // x alignment in cells
  static constexpr int NA = 32;
  // x extent: along x the 32-cell line plus the shift of the rounded start;
  // across x the NC lines, whose tiles start at multiples of NC cells
  static_assert(DIR == 0 || NC % XA == 0, "tiles across x start on 16-byte boundaries");
  static constexpr int BX = DIR == 0 ? (NA + XA - 1 + XA - 1) / XA * XA : NC;
  static constexpr int BY = DIR == 0 ? NC : (DIR == 1 ? NA : 1);
  static constexpr int BZ = DIR == 2 ? NA : 1;
  static constexpr int CELLS = BX * BY * BZ;
  static constexpr unsigned BYTES5 = (unsigned)(CELLS * 5 * sizeof(R));
  static constexpr unsigned BYTES9 = (unsigned)(CELLS * 9 * sizeof(R));
  // the second box starts on a 128-byte boundary
  static constexpr int OFF9 = (int)((BYTES5 + 127) / 128 * 128 / sizeof(R));
  static constexpr size_t SPAN = (size_t)OFF9 * sizeof(R) + BYTES9;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// bounded wait for phase 0 of the barrier; false if it did not complete
__device__ __forceinline__ bool mbar_wait0(unsigned long long* bar, int max_polls) {
  for (int k = 0; k < max_polls; k++) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(0u)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int f,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(f), "r"(smem_u32(bar))
      : "memory");
}

// weno_lr_pair across a warp (FP64): lane a reconstructs both face states of
// the two quantities of pair array q at line position s.  Neighbouring
// stencils share terms: the second difference a lane centres on itself is
// the one the stencil of lane a-1 needs on its right and lane a+1 on its
// left, and the candidate polynomials 2q_j + 5q_{j+1} - q_{j+2} and
// -q_{j-1} + 5q_j + 2q_{j+1} of lane a-1's left face are lane a's right-face
// candidates; each is formed once and passed by shuffle.  Every lane of the
// warp calls this (the stencil positions are clamped to the line, so lanes
// whose stencil leaves it form values that nobody uses).  Same weights and
// single reciprocal as weno_lr_pair.
__device__ __forceinline__ void weno_lr_pair_warp(const double (*q)[2], int s, int a, double& La, double& Ra,
                                                  double& Lb, double& Rb) {
  const int lo = s - a, hi = s - a + 31;
  double x[5][2];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    int i = s - 2 + k;
    i = (i < lo || i > hi) ? s : i;
    const double2 v = ld_pair(q, i);
    x[k][0] = v.x;
    x[k][1] = v.y;
  }
  const double c13 = 13. / 12., eps = 1e-6;
  double num[4], den[4];
#pragma unroll
  for (int m = 0; m < 2; m++) {
    const double qm2 = x[0][m], qm1 = x[1][m], qc = x[2][m], qp1 = x[3][m], qp2 = x[4][m];
    // the squared second difference centred on this lane, and the ones
    // centred on the neighbours
    const double d1 = qm1 - 2 * qc + qp1, s1 = d1 * d1;
    const double s0 = __shfl_down_sync(0xffffffffu, s1, 1), s2 = __shfl_up_sync(0xffffffffu, s1, 1);
    const double g0 = 3 * qc - 4 * qp1 + qp2, g1 = qm1 - qp1, g2 = qm2 - 4 * qm1 + 3 * qc;
    const double b0 = fma(c13, s0, 0.25 * (g0 * g0)), b1 = fma(c13, s1, 0.25 * (g1 * g1)),
                 b2 = fma(c13, s2, 0.25 * (g2 * g2));
    const double e0 = eps + b0, e1 = eps + b1, e2 = eps + b2;
    const double E0 = e0 * e0, E1 = e1 * e1, E2 = e2 * e2;
    const double P12 = E1 * E2, P02 = E0 * E2, P01 = E0 * E1;
    const double nl0 = 0.3 * P12, nl1 = 0.6 * P02, nl2 = 0.1 * P01;
    const double nr0 = 0.1 * P12, nr1 = nl1, nr2 = 0.3 * P01;
    const double ql0 = 2 * qc + 5 * qp1 - qp2;
    const double ql1 = -qm1 + 5 * qc + 2 * qp1;
    const double ql2 = 2 * qm2 - 7 * qm1 + 11 * qc;
    const double qr0 = 11 * qc - 7 * qp1 + 2 * qp2;
    const double qr1 = __shfl_up_sync(0xffffffffu, ql0, 1);  // 2 q_{a-1} + 5 q_a - q_{a+1}
    const double qr2 = __shfl_up_sync(0xffffffffu, ql1, 1);  // -q_{a-2} + 5 q_{a-1} + 2 q_a
    num[2 * m] = nl0 * ql0 + nl1 * ql1 + nl2 * ql2;
    den[2 * m] = 6 * (nl0 + nl1 + nl2);
    num[2 * m + 1] = nr0 * qr0 + nr1 * qr1 + nr2 * qr2;
    den[2 * m + 1] = 6 * (nr0 + nr1 + nr2);
  }
  const double d01 = den[0] * den[1], d23 = den[2] * den[3];
  const double inv = 1.0 / (d01 * d23);
  const double i01 = d23 * inv, i23 = d01 * inv;
  La = num[0] * den[1] * i01;
  Ra = num[1] * den[0] * i01;
  Lb = num[2] * den[3] * i23;
  Rb = num[3] * den[2] * i23;
}

template <class R>
__device__ inline R shfl_dn(R v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }
template <class R>
__device__ inline R shfl_up(R v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }

// One tile of the flux sweep along DIR: tile index bx along the direction,
// by across it, bz the third axis (interior index).  NC*32 threads.
template <class R, int DIR, int NC, int UNR = 1, bool TMA = false>
__device__ __forceinline__ void dir_tile(const DevCfg& C, const DevPtrs<R>& P, int use_b, R tau, R inv_h, R h,
                                         int first, int bx, int by, int bz, DirSmem<R, DIR, NC>& sm,
                                         const CUtensorMap* map5 = nullptr, const CUtensorMap* map9 = nullptr) {
  using S = DirSmem<R, DIR, NC>;
  constexpr int NA = S::NA, TL = S::TL, LD = S::LD;
  static_assert(NA == 32, "one warp per line");
  const int tid = threadIdx.x;
  int lo, hi, galong;
  if (DIR == 0) { lo = C.il; hi = C.ir; galong = C.gx; }
  else if (DIR == 1) { lo = C.jl; hi = C.jr; galong = C.gy; }
  else { lo = C.kl; hi = C.kr; galong = C.gz; }
  const int a0 = lo - NG + bx * TL;  // global along index of local 0
  const long long stride = DIR == 0 ? 1 : (DIR == 1 ? (long long)C.px : (long long)C.px * C.gy);

  // cross coordinates of line c.  Across x (the y and eta sweeps) the
  // tiles start at x = xt0 + by * NC: on a handle's padded rows xt0 = 0, so
  // that a tile's x segment sits on whole 32-byte sectors (the lines in the
  // ghost cells are idle); on unpadded rows xt0 = il.
  auto cross_base = [&](int c, bool& ok) -> long long {
    int i, j, k;
    if (DIR == 0) { i = 0; j = C.jl + by * NC + c; k = C.kl + bz; ok = j < C.jr; }
    else if (DIR == 1) { i = C.xt0 + by * NC + c; j = 0; k = C.kl + bz; ok = i >= C.il && i < C.ir; }
    else { i = C.xt0 + by * NC + c; j = C.jl + bz; k = 0; ok = i >= C.il && i < C.ir; }
    return cix(C, i, j, k);
  };

      // ---- load and per-cell terms (x-fastest thread order: coalesced)
  {
    const int ta = DIR == 0 ? tid % NA : tid / NC;
    const int tc = DIR == 0 ? tid / NA : tid % NC;
    bool ok;
    const long long cb = cross_base(tc, ok);
    const int g = a0 + ta;
    const int s = tc * LD + ta;
    R F[9], V[9], spd = 0, uu[4] = {0, 0, 0, 0};
    const bool live = ok && g >= 0 && g < galong;
    R e = 0, p[5], T[4];  // the TMA path's copy of the cell
    if constexpr (TMA) {
      // the tile arrives by two box copies into the front of the shared
      // buffer (the flux arrays overwrite it after the barrier below)
      using B = TmaBox<R, DIR, NC>;
      static_assert(B::SPAN <= sizeof(DirSmem<R, DIR, NC>), "staging fits");
      __shared__ __align__(8) unsigned long long bar;
      R* raw = reinterpret_cast<R*>(&sm);
      const int xc = DIR == 0 ? a0 : C.xt0 + by * NC;  // first x of the tile
      const int x0 = xc / B::XA * B::XA;               // rounded down to 16 bytes
      const int y0 = DIR == 0 ? C.jl + by * NC : (DIR == 1 ? a0 : C.jl + bz);
      const int z0 = DIR == 2 ? a0 : C.kl + bz;
      // a box lands only on a 128-byte boundary of shared memory (the same
      // address in every thread: the block leaves as a whole)
      if (smem_u32(raw) & 127u) {
        if (tid == 0) atomicOr(P.status, ST_TMA);
        return;
      }
      if (tid == 0) mbar_init(&bar, 1);
      __syncthreads();
      if (tid == 0) {
        mbar_expect_tx(&bar, B::BYTES5 + B::BYTES9);
        tma_load_4d(raw, map5, x0, y0, z0, 0, &bar);
        tma_load_4d(raw + B::OFF9, map9, x0, y0, z0, use_b ? 18 : 5, &bar);
      }
      // every thread waits for the copies (bounded); the block leaves as a
      // whole if any of them gave up, after a second bounded wait for the
      // copies still in flight, with the step flagged
      const bool got = mbar_wait0(&bar, 1 << 22);
      if (!__syncthreads_and(got)) {
        if (tid == 0) atomicOr(P.status, ST_TMA);
        mbar_wait0(&bar, 1 << 22);
        return;
      }
      const int xl = DIR == 0 ? ta + (xc - x0) : tc + (xc - x0);
      const int yl = DIR == 1 ? ta : (DIR == 0 ? tc : 0);
      const int zl = DIR == 2 ? ta : 0;
      const int o = (zl * B::BY + yl) * B::BX + xl;
      if (live) {
        e = raw[o];
#pragma unroll
        for (int l = 0; l < 4; l++) uu[l] = raw[(1 + l) * B::CELLS + o];
        const R* c9 = raw + B::OFF9 + o;
#pragma unroll
        for (int l = 0; l < 4; l++) T[l] = c9[(use_b ? l : 5 + l) * B::CELLS];
#pragma unroll
        for (int l = 0; l < 5; l++) p[l] = c9[(use_b ? 4 + l : l) * B::CELLS];
      }
      __syncthreads();  // every thread has its cell before the buffer is reused
      if (live) {
        cell_terms<R, DIR>(C, tau, e, uu, p, T, g >= lo && g < hi, F, V, spd);
      } else {
#pragma unroll
        for (int l = 0; l < 9; l++) { F[l] = 0; V[l] = 0; }
      }
    } else if (live) {
      const long long c = cb + (long long)g * stride;
      R p2[5], T2[4];
      const R e2 = P.e()[c];
#pragma unroll
      for (int l = 0; l < 4; l++) uu[l] = P.u(l)[c];
#pragma unroll
      for (int l = 0; l < 4; l++) T2[l] = P.S(use_b, l)[c];
#pragma unroll
      for (int l = 0; l < 5; l++) p2[l] = P.S(use_b, 4 + l)[c];
      cell_terms<R, DIR>(C, tau, e2, uu, p2, T2, g >= lo && g < hi, F, V, spd);
    } else {
#pragma unroll
      for (int l = 0; l < 9; l++) { F[l] = 0; V[l] = 0; }
    }
#pragma unroll
    for (int l = 0; l < 9; l++) { sm.fv[l][s][0] = F[l]; sm.fv[l][s][1] = V[l]; }
    sm.spd[s] = spd;
#pragma unroll
    for (int l = 0; l < 4; l++) sm.up[l >> 1][s][l & 1] = uu[l];
  }
  __syncthreads();

  // ---- one warp per line: lane a reconstructs both face states of its
  // stencil; the face right of lane a takes R from lane a + 1.
  // Along x the lanes of a warp are consecutive cells and write the
  // divergence and the velocity derivative straight to the state arrays.
  // Across x (TR) a warp's cells are a row apart; each warp leaves its
  // results in its own line of shared memory (the slots its stencil has
  // finished reading) and the block writes them row by row at the end.
  constexpr bool TR = DIR != 0;
  const int a = tid & 31, c = tid >> 5;
  bool ok;
  const long long cb = cross_base(c, ok);
  if (!TR && !ok) return;  // whole warp: c is uniform in the warp (no barrier follows)
  const int g = a0 + a;
  const int s = c * LD + a;
  const bool stencil = a >= 2 && a <= NA - 3;  // a-2..a+2 inside the tile
  const bool out = a >= 3 && a < 3 + TL && g < hi;  // interior cell of this tile
  const long long cell = cb + (long long)g * stride;
  if (ok) {
    // face right of lane a exists for lanes 2..NA-4; it is a needed face
    // when the cell right of it is in [lo, hi]
    R amax = 0;
    {
      R L = 0, Rr = 0;
      if (stencil) recon_lr<R>(C, sm.spd, s, L, Rr);
      const R Rn = shfl_dn<R>(Rr, 1);
      // the face left of the first interior cell takes no dissipation: its
      // max speed sits in a ghost cell the reference never fills
      // (NEWEST5/hydroKT.h:265-314 vs 435-440)
      amax = (g + 1 == lo) ? (R)0 : fmax(fabs(L), fabs(Rn));
    }
    // the divergence accumulated by the previous sweeps: loaded before the
    // flux loop so that the loads overlap the reconstruction
    R racc[9];
#pragma unroll
    for (int l = 0; l < 9; l++) racc[l] = (!TR && !first && out) ? P.res(l)[cell] : (R)0;
#pragma unroll UNR
    for (int l = 0; l < 9; l++) {
      R fl = 0, fr = 0, vl = 0, vr = 0;
      if (stencil) {
        if constexpr (sizeof(R) == 4) {
          if (C.recon == 0) {
            // F^l and V^l of the stencil reconstructed as one pair
            const float(*q)[2] = reinterpret_cast<const float(*)[2]>(sm.fv[l]);
            F2 L2, R2, x0, x1, x2, x3, x4;
            x0.v = ld_pair(q, s - 2); x1.v = ld_pair(q, s - 1); x2.v = ld_pair(q, s);
            x3.v = ld_pair(q, s + 1); x4.v = ld_pair(q, s + 2);
            weno_lr2(x0, x1, x2, x3, x4, L2, R2);
            float a, b;
            f2u(L2, a, b);
            fl = a; vl = b;
            f2u(R2, a, b);
            fr = a; vr = b;
          } else {
            recon_lr<R, 2>(C, &sm.fv[l][0][0], s, fl, fr);
            recon_lr<R, 2>(C, &sm.fv[l][0][1], s, vl, vr);
          }
        } else if (C.recon != 0) {
          recon_lr<R, 2>(C, &sm.fv[l][0][0], s, fl, fr);
          recon_lr<R, 2>(C, &sm.fv[l][0][1], s, vl, vr);
        }
      }
      if constexpr (sizeof(R) == 8) {
        if (C.recon == 0) {
          // F^l and V^l with one reciprocal between them; every lane takes
          // part (the stencils' shared terms travel by shuffle)
          double flx, frx, vlx, vrx;
          weno_lr_pair_warp(reinterpret_cast<const double(*)[2]>(sm.fv[l]), s, a, flx, frx, vlx, vrx);
          if (stencil) { fl = flx; fr = frx; vl = vlx; vr = vrx; }
        }
      }
      fr = shfl_dn<R>(fr, 1);
      vr = shfl_dn<R>(vr, 1);
      const R H = (R)0.5 * (fl + fr) - (R)0.5 * amax * (vr - vl);  // flux at the right face
      const R Hl = shfl_up<R>(H, 1);                                // flux at the left face
      const R r = -inv_h * (H - Hl);
      if constexpr (TR) {
        __syncwarp();  // the line's stencil reads of field l are done
        if (out) sm.fv[l][s][0] = r;
      } else if (out) {
        P.res(l)[cell] = first ? r : racc[l] + r;
      }
    }
    // velocity derivative along DIR: (L - R)/h of the same stencil (genWENOder)
    R dv[4] = {0, 0, 0, 0};
#pragma unroll
    for (int l = 0; l < 4; l += 2) {
      R La = 0, Ra = 0, Lb = 0, Rb = 0;
      if constexpr (sizeof(R) == 4) {
        if (out) {
          const float(*q)[2] = reinterpret_cast<const float(*)[2]>(sm.up[l >> 1]);
          F2 L2, R2, x0, x1, x2, x3, x4;
          x0.v = ld_pair(q, s - 2); x1.v = ld_pair(q, s - 1); x2.v = ld_pair(q, s);
          x3.v = ld_pair(q, s + 1); x4.v = ld_pair(q, s + 2);
          weno_lr2(x0, x1, x2, x3, x4, L2, R2);
          f2u(L2, La, Lb);
          f2u(R2, Ra, Rb);
        }
      } else {
        // every lane takes part (shuffles); the out lanes keep the result
        weno_lr_pair_warp(reinterpret_cast<const double(*)[2]>(sm.up[l >> 1]), s, a, La, Ra, Lb, Rb);
      }
      if (out) {
        dv[l] = (La - Ra) * inv_h;
        dv[l + 1] = (Lb - Rb) * inv_h;
      }
    }
    if constexpr (TR) {
      __syncwarp();  // the line's velocity stencils are read
      if (out) {
#pragma unroll
        for (int l = 0; l < 4; l++) sm.up[l >> 1][s][l & 1] = dv[l];
      }
    } else if (out) {
#pragma unroll
      for (int l = 0; l < 4; l++) P.du(l * 3 + DIR)[cell] = dv[l];
    }
  }
  if constexpr (TR) {
    __syncthreads();
    // row by row: x fastest (along the line for x, over the tile's NC lines
    // across x)
    for (int t = tid; t < NC * TL; t += NC * NA) {
      const int cc = DIR == 0 ? t / TL : t % NC, aa = 3 + (DIR == 0 ? t % TL : t / NC);
      bool ok2;
      const long long cb2 = cross_base(cc, ok2);
      const int g2 = a0 + aa;
      if (!ok2 || g2 >= hi) continue;
      const long long cell2 = cb2 + (long long)g2 * stride;
      const int s2 = cc * LD + aa;
      R acc[9];
#pragma unroll
      for (int l = 0; l < 9; l++) acc[l] = first ? (R)0 : P.res(l)[cell2];
#pragma unroll
      for (int l = 0; l < 9; l++) P.res(l)[cell2] = first ? sm.fv[l][s2][0] : acc[l] + sm.fv[l][s2][0];
#pragma unroll
      for (int l = 0; l < 4; l++) P.du(l * 3 + DIR)[cell2] = sm.up[l >> 1][s2][l & 1];
    }
  }
}

// Blocks per SM the sweeps are compiled for.  FP64: 4 blocks of 256
// threads (y, eta) and 7 of 128 (x) hold the registers to 64 and 72 a
// thread, a few bytes of spill in the y and eta sweeps against a fourth
// resident block (measured: the FP64 step 2 % faster than at 3 blocks and
// 80 registers).  FP32: the counts the registers the sweeps need allow
// anyway (48 a thread; 40 for the y and eta sweeps staged by TMA).
template <class R, int DIR, bool TMA>
struct DirOcc {
  static constexpr int MIN_BLOCKS = sizeof(R) == 8 ? (DIR == 0 ? 7 : 4) : (DIR == 0 ? 10 : (TMA ? 6 : 5));
};

// the sweep with its tile staged by TMA (the handle's padded state)
template <class R, int DIR>
__global__ void __launch_bounds__(Tile<DIR, R>::NA* Tile<DIR, R>::NC, DirOcc<R, DIR, true>::MIN_BLOCKS)
    k_dir_tma(DevCfg C, DevPtrs<R> P, int use_b, R tau, R inv_h, R h, int first,
              const __grid_constant__ CUtensorMap map5, const __grid_constant__ CUtensorMap map9) {
  using S = DirSmem<R, DIR>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  pdl_wait_then_release();
  if (*P.status) return;
  dir_tile<R, DIR, S::NC, 1, true>(C, P, use_b, tau, inv_h, h, first, blockIdx.x, blockIdx.y, blockIdx.z,
                                   *reinterpret_cast<S*>(smem_raw), &map5, &map9);
}

template <class R, int DIR>
__global__ void __launch_bounds__(Tile<DIR, R>::NA* Tile<DIR, R>::NC, DirOcc<R, DIR, false>::MIN_BLOCKS)
    k_dir(DevCfg C, DevPtrs<R> P, int use_b, R tau, R inv_h, R h, int first) {
  using S = DirSmem<R, DIR>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  pdl_wait_then_release();
  if (*P.status) return;
  dir_tile<R, DIR, S::NC>(C, P, use_b, tau, inv_h, h, first, blockIdx.x, blockIdx.y, blockIdx.z,
                          *reinterpret_cast<S*>(smem_raw));
}

// Copy one cell's fields into a ghost cell (NEWEST5/boundary.h).
template <class R>
__device__ inline void ghost_put(const DevPtrs<R>& P, int set_b, long long dst, R e, const R* u, const R* pu,
                                 const R* q9, bool skip_u12) {
  P.e()[dst] = e;
  P.u(0)[dst] = u[0];
  if (!skip_u12) { P.u(1)[dst] = u[1]; P.u(2)[dst] = u[2]; }
  P.u(3)[dst] = u[3];
#pragma unroll
  for (int l = 0; l < 4; l++) P.pu(l)[dst] = pu[l];
#pragma unroll
  for (int l = 0; l < 9; l++) P.S(set_b, l)[dst] = q9[l];
}

// The update of one interior cell, in two parts: rk_cell (du_tau, sources,
// the RK combination, prevu) and root_cell (the root-find and the ghost
// copy).  STAGE 1 reads set A and writes set B and v1t; STAGE 2 reads A (its
// own cell), B and v1t and writes A.
struct CellAt {
  int i, j, k;
  long long c;
};
__device__ __forceinline__ CellAt cell_at(const DevCfg& C, long long t) {
  CellAt x;
  x.i = C.il + (int)(t % C.nx);
  x.j = C.jl + (int)((t / C.nx) % C.ny);
  x.k = C.kl + (int)(t / ((long long)C.nx * C.ny));
  x.c = cix(C, x.i, x.j, x.k);
  return x;
}

// Sources and RK combination of cell x: stores the new conserved set (q9,
// also returned) and, at stage 1, v1t and prevu; returns e, u and prevu for
// the root-find.
template <class R, int STAGE>
__device__ __forceinline__ void rk_cell(const DevCfg& C, const DevPtrs<R>& P, double tau_n, double ts, const CellAt& x,
                                        R& e_out, R* u_out, R* pu_out, R* q9) {
  {
    const int k = x.k;
    const long long c = x.c;
    const double tau1 = tau_n + ts;
    const R tau_s = (R)(STAGE == 1 ? tau_n : tau1);  // time of the sources
    const bool cart = C.cart;

    R u[4], pu[4], p[5], e = P.e()[c];
#pragma unroll
    for (int l = 0; l < 4; l++) { u[l] = P.u(l)[c]; pu[l] = P.pu(l)[c]; }
    const int cur_b = STAGE == 1 ? 0 : 1;  // conserved set read
    R Tc[4];
#pragma unroll
    for (int l = 0; l < 4; l++) Tc[l] = P.S(cur_b, l)[c];
#pragma unroll
    for (int l = 0; l < 5; l++) p[l] = P.S(cur_b, 4 + l)[c];

    // velocity gradients
    R du[4][4];
#pragma unroll
    for (int l = 0; l < 4; l++) {
      du[l][0] = (u[l] - pu[l]) * (R)(1.0 / ts);
      du[l][1] = P.du(l * 3 + 0)[c];
      du[l][2] = P.du(l * 3 + 1)[c];
      du[l][3] = C.bi ? (R)0 : P.du(l * 3 + 2)[c];
    }
    // sources (NEWEST5/Source.h:165-191 geometric, 311-433 shear)
    R src[9];
    {
      R Pp, cs2, Te;
      eos_all<R>(C, e, Pp, cs2, Te);
      if (cart) {
        src[0] = src[1] = src[2] = src[3] = 0;
      } else {
        const R t2 = tau_s * tau_s;
        PiDep<R> d = pi_dep<R>(u[0], u[1], u[2], u[3], p, t2);
        const R ep = e + Pp;
        src[0] = -Pp - t2 * (d.ee + ep * u[3] * u[3]);
        src[1] = 0;
        src[2] = 0;
        src[3] = -(R)2 * (d.te + ep * u[0] * u[3]);
      }
      R s5[5];
      is_source_PT<R>(C, tau_s, e, Pp, Te, u, p, du, s5);
      // TXYZ5/Source.h:268-270: the Cartesian 3+1D shear source skips the
      // last three interior z layers
      if (cart && !C.bi && (k - C.kl) >= C.nz - NG) s5[0] = s5[1] = s5[2] = s5[3] = s5[4] = 0;
#pragma unroll
      for (int q = 0; q < 5; q++) src[4 + q] = s5[q];
    }
    // RK combination (NEWEST5/time.h:2-140)
    R Vn[9];
    const int out_b = STAGE == 1 ? 1 : 0;  // conserved set written
    if (STAGE == 1) {
#pragma unroll
      for (int l = 0; l < 9; l++) {
        const R L0 = P.res(l)[c] + src[l];
        const R v0 = l < 4 ? (cart ? Tc[l] : (R)tau_n * Tc[l]) : p[l - 4];
        Vn[l] = v0 + (R)ts * L0;
      }
#pragma unroll
      for (int l = 0; l < 4; l++) P.v1t(l)[c] = Vn[l];
    } else {
#pragma unroll
      for (int l = 0; l < 9; l++) {
        const R L1 = P.res(l)[c] + src[l];
        const R v0 = l < 4 ? (cart ? P.A(l)[c] : (R)tau_n * P.A(l)[c]) : P.A(l)[c];
        const R v1 = l < 4 ? P.v1t(l)[c] : p[l - 4];
        Vn[l] = (R)0.5 * v0 + (R)0.5 * v1 + (R)0.5 * (R)ts * L1;
      }
    }
#pragma unroll
    for (int l = 0; l < 4; l++) q9[l] = cart ? Vn[l] : Vn[l] * (R)(1.0 / tau1);
#pragma unroll
    for (int l = 0; l < 5; l++) q9[4 + l] = Vn[4 + l];
#pragma unroll
    for (int l = 0; l < 9; l++) P.S(out_b, l)[c] = q9[l];
    // the root-find's first start: e scaled by the change of T^{tau tau}
    // and, at stage 1, the velocity extrapolated linearly from prevu (the
    // root is the same; root_cell falls back to the stage's primitives)
    const R rt = q9[0] / Tc[0];
    e_out = (rt > (R)0.5 && rt < (R)2) ? e * rt : e;
    u_out[0] = u[0];
#pragma unroll
    for (int l = 1; l < 4; l++) u_out[l] = STAGE == 1 ? (R)2 * u[l] - pu[l] : u[l];
    // previous velocity (NEWEST5/time.h:166, stage 1 only)
    if (STAGE == 1) {
#pragma unroll
      for (int l = 0; l < 4; l++) { pu[l] = u[l]; P.pu(l)[c] = u[l]; }
    }
#pragma unroll
    for (int l = 0; l < 4; l++) pu_out[l] = pu[l];
  }
}

// Root-find (FP64) of cell x from its new conserved set q9 with (e, u) as the
// guess, then the ghost copy; returns the Newton iterations and, at stage 2,
// the new temperature in GeV in *t_gev.
template <class R, int STAGE>
__device__ __forceinline__ unsigned root_cell(const DevCfg& C, const DevPtrs<R>& P, double tau_n, double ts,
                                              const CellAt& at, R e, R* u, const R* pu, const R* q9, double* t_gev) {
  unsigned my_it = 0;
  {
    const int i = at.i, j = at.j, k = at.k;
    const long long c = at.c;
    const double tau1 = tau_n + ts;
    const bool cart = C.cart;
    const int out_b = STAGE == 1 ? 1 : 0;  // conserved set written
    // root-find (FP64) with the current primitives as the guess
    double Tt[4], pd[5], x[4] = {(double)e, (double)u[1], (double)u[2], (double)u[3]};
#pragma unroll
    for (int l = 0; l < 4; l++) Tt[l] = (double)q9[l];
#pragma unroll
    for (int l = 0; l < 5; l++) pd[l] = (double)q9[4 + l];
    // stopping (con2prim): FP64 steps below 1e-13, or an undamped one below
    // 1e-8, taken without the confirming evaluation; the mixed mode stores
    // the result in FP32, so a Newton step below 3e-4 ends it (the error it
    // leaves, of the order of its square, is below FP32 rounding)
    const double rtol = sizeof(R) == 4 ? 1e-10 : 1e-13, qtol = sizeof(R) == 4 ? 1e-6 : 1e-8;
    const double qskip = sizeof(R) == 4 ? 3e-4 : 1e-8, fskip = sizeof(R) == 4 ? 3e-3 : 1e-6;
    int it = -1;
    // a second attempt starts from the stage's primitives, still in memory
    // (near-vacuum cells, where the extrapolated start can lead Newton
    // astray); one loop keeps a single copy of the solver in the kernel
#pragma unroll 1
    for (int attempt = 0; attempt < 2 && it < 0; attempt++) {
      if (attempt) {
        x[0] = (double)P.e()[c];
#pragma unroll
        for (int l = 1; l < 4; l++) x[l] = (double)P.u(l)[c];
      }
      it = con2prim(C, Tt, pd, tau1, x, rtol, qtol, qskip, fskip);
    }
    if (it < 0) {
      atomicOr(P.status, ST_ROOT);
    } else {
      my_it = (unsigned)it;
      const double tt = cart ? 1.0 : tau1;
      const double u0 = sqrt(1 + x[1] * x[1] + x[2] * x[2] + x[3] * x[3] * tt * tt);
      const double vx = x[1] / u0, vy = x[2] / u0, ve = x[3] / u0;
      if (sqrt(vx * vx + vy * vy + tt * tt * ve * ve) >= 1) atomicOr(P.status, ST_CAUSAL);
      if (x[0] <= 0) atomicOr(P.status, ST_NEGE);
      e = (R)x[0];
      u[0] = (R)u0; u[1] = (R)x[1]; u[2] = (R)x[2]; u[3] = (R)x[3];
      P.e()[c] = e;
#pragma unroll
      for (int l = 0; l < 4; l++) P.u(l)[c] = u[l];
    }
    // ghost copy of boundary cells: faces only, corners untouched
    // (NEWEST5/boundary.h:1-276); Gubser test mirrors u^x,u^y.  A boundary
    // cell reads back the conserved set and prevu it stored above, so that
    // they need not stay in registers through the root-find.
    const bool mir = C.mirror;
    const bool edge = i == C.il || i == C.ir - 1 || j == C.jl || j == C.jr - 1 || (!C.bi && (k == C.kl || k == C.kr - 1));
    const bool near = mir && (i - C.il < NG || C.ir - 1 - i < NG || j - C.jl < NG || C.jr - 1 - j < NG);
    if (!edge && !near) {
      if (STAGE == 2 && t_gev) *t_gev = C.hbarc * (double)eos_T<R>(C, e);
      return my_it;
    }
    R qb[9], pb[4];
    if (edge) {
#pragma unroll
      for (int l = 0; l < 9; l++) qb[l] = P.S(out_b, l)[c];
#pragma unroll
      for (int l = 0; l < 4; l++) pb[l] = P.pu(l)[c];
    }
    q9 = qb;
    pu = pb;
    if (i == C.il)
      for (int m = 0; m < NG; m++) ghost_put<R>(P, out_b, cix(C, m, j, k), e, u, pu, q9, mir);
    if (i == C.ir - 1)
      for (int m = 0; m < NG; m++) ghost_put<R>(P, out_b, cix(C, C.ir + m, j, k), e, u, pu, q9, mir);
    if (j == C.jl)
      for (int m = 0; m < NG; m++) ghost_put<R>(P, out_b, cix(C, i, m, k), e, u, pu, q9, mir);
    if (j == C.jr - 1)
      for (int m = 0; m < NG; m++) ghost_put<R>(P, out_b, cix(C, i, C.jr + m, k), e, u, pu, q9, mir);
    if (!C.bi) {
      if (k == C.kl)
        for (int m = 0; m < NG; m++) ghost_put<R>(P, out_b, cix(C, i, j, m), e, u, pu, q9, false);
      if (k == C.kr - 1)
        for (int m = 0; m < NG; m++) ghost_put<R>(P, out_b, cix(C, i, j, C.kr + m), e, u, pu, q9, false);
    }
    if (mir) {
      // ghost m <- cell il + 2 - m on the left, ghost ir + m <- ir - 1 - m on the right
      const int dl = i - C.il, dr = C.ir - 1 - i;
      if (dl < NG) { long long g = cix(C, C.il - 1 - dl, j, k); P.u(1)[g] = u[1]; P.u(2)[g] = u[2]; }
      if (dr < NG) { long long g = cix(C, C.ir + dr, j, k); P.u(1)[g] = u[1]; P.u(2)[g] = u[2]; }
      const int el = j - C.jl, er = C.jr - 1 - j;
      if (el < NG) { long long g = cix(C, i, C.jl - 1 - el, k); P.u(1)[g] = u[1]; P.u(2)[g] = u[2]; }
      if (er < NG) { long long g = cix(C, i, C.jr + er, k); P.u(1)[g] = u[1]; P.u(2)[g] = u[2]; }
    }
    if (STAGE == 2 && t_gev) *t_gev = C.hbarc * (double)eos_T<R>(C, e);
  }
  return my_it;
}

// One interior cell t (0 <= t < nx*ny*nz) of the update, both parts.
template <class R, int STAGE>
__device__ __forceinline__ unsigned update_cell(const DevCfg& C, const DevPtrs<R>& P, double tau_n, double ts,
                                                long long t, double* t_gev) {
  const CellAt x = cell_at(C, t);
  R e, u[4], pu[4], q9[9];
  rk_cell<R, STAGE>(C, P, tau_n, ts, x, e, u, pu, q9);
  return root_cell<R, STAGE>(C, P, tau_n, ts, x, e, u, pu, q9, t_gev);
}

// one thread per interior cell.  Blocks per SM: FP64 4 (128 registers),
// mixed 5 (96 registers); measured on the 161x161x41 event, FP64 per step
// 1.671 / 1.719 / 1.775 / 1.797 ms at 4 / 5 / 6 / 7 blocks (fewer spills
// win), mixed 0.975 / 0.957 / 0.977 / 0.977 ms
template <class R>
struct UpdOcc {
  static constexpr int MIN_BLOCKS = sizeof(R) == 8 ? 4 : 5;
};
template <class R, int STAGE>
__global__ void __launch_bounds__(128, UpdOcc<R>::MIN_BLOCKS) k_update(DevCfg C, DevPtrs<R> P, double tau_n, double ts) {
  pdl_wait_then_release();
  if (*P.status) return;
  const long long nint = (long long)C.nx * C.ny * (C.kr - C.kl);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long my_it = t < nint ? update_cell<R, STAGE>(C, P, tau_n, ts, t, nullptr) : 0u;
  // one atomic per warp for the iteration counter
  for (int o = 16; o > 0; o >>= 1) my_it += __shfl_down_sync(0xffffffffu, my_it, o);
  if ((threadIdx.x & 31) == 0 && my_it) atomicAdd(P.iters, my_it);
}

}  // namespace vh
