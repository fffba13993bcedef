// C ABI of the B200 viscous KT step (include/vh.h): handle, device buffers,
// state transfer, the TVDRK2 step loop and the reductions.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <string>
#include <vector>

#include "vh.h"
#include "vh_handle.cuh"
#include "vh_internal.h"

using namespace vh;


static std::string g_create_err;

static int validate(const vh_config* c, std::string& why) {
  if (!c) { why = "null config"; return VH_E_ARG; }
  if (c->coords != VH_COORD_MILNE && c->coords != VH_COORD_CARTESIAN) { why = "coords"; return VH_E_ARG; }
  if (c->precision != VH_PREC_FP64 && c->precision != VH_PREC_MIXED) { why = "precision"; return VH_E_ARG; }
  if (c->recon != VH_RECON_WENO5 && c->recon != VH_RECON_MINMOD) { why = "recon"; return VH_E_ARG; }
  if (c->nx < 3 || c->ny < 3 || (!c->boost_invariant && c->nz < 3)) { why = "grid needs >= 3 interior cells per axis"; return VH_E_ARG; }
  if (c->boost_invariant && c->nz != 1) { why = "boost-invariant grids have nz = 1"; return VH_E_ARG; }
  if (!(c->dx > 0 && c->dy > 0 && (c->boost_invariant || c->dz > 0))) { why = "cell sizes"; return VH_E_ARG; }
  if (!(c->dtau > 0) || (c->coords == VH_COORD_MILNE && !(c->tau0 > 0))) { why = "tau0/dtau"; return VH_E_ARG; }
  if (c->eos_kind == VH_EOS_CONFORMAL) {
    if (!(c->eos_a > 0)) { why = "eos_a"; return VH_E_ARG; }
  } else if (c->eos_kind == VH_EOS_TABLE) {
    if (c->eos_n < 2 || !c->eos_e || !c->eos_p || !c->eos_cs2 || !c->eos_t) { why = "eos table"; return VH_E_ARG; }
    for (int i = 1; i < c->eos_n; i++)
      if (!(c->eos_e[i] > c->eos_e[i - 1])) { why = "eos table e must increase"; return VH_E_ARG; }
  } else { why = "eos_kind"; return VH_E_ARG; }
  if (c->taupi_kind != VH_TAUPI_15_ETA_OVER_P && c->taupi_kind != VH_TAUPI_5_ETA_OVER_EPP &&
      c->taupi_kind != VH_TAUPI_CONST) { why = "taupi_kind"; return VH_E_ARG; }
  if (c->taupi_kind == VH_TAUPI_CONST && !(c->taupi_const > 0)) { why = "taupi_const"; return VH_E_ARG; }
  return VH_OK;
}

extern "C" int vh_create(const vh_config* cfg, vh_handle** out) {
  std::string why;
  if (!out) return VH_E_ARG;
  *out = nullptr;
  int v = validate(cfg, why);
  if (v != VH_OK) { g_create_err = "vh_create: " + why; return v; }
  vh_handle* h = new vh_handle();
  h->cfg = *cfg;
  h->cfg.eos_e = h->cfg.eos_p = h->cfg.eos_cs2 = h->cfg.eos_t = nullptr;
  h->mixed = cfg->precision == VH_PREC_MIXED;
  h->esz = h->mixed ? 4 : 8;
  DevCfg& C = h->C;
  C.nx = cfg->nx; C.ny = cfg->ny; C.nz = cfg->boost_invariant ? 1 : cfg->nz;
  C.gx = cfg->nx + 2 * NG; C.gy = cfg->ny + 2 * NG; C.gz = cfg->boost_invariant ? 1 : cfg->nz + 2 * NG;
  // rows padded to a multiple of 8 cells (32 bytes in FP32, 64 in FP64), so
  // that every row of every array starts on a 32-byte sector: the y and eta
  // sweeps' tiles (8 lines across x, starting at multiples of 8 cells) then
  // read and write whole sectors, and the TMA tiles' strides are multiples
  // of 16 bytes as the tensor maps require.  The padding cells are never
  // read; the C ABI's arrays keep the canonical unpadded layout.
  C.px = (C.gx + 7) / 8 * 8;
  C.xt0 = 0;
  C.il = NG; C.ir = NG + cfg->nx; C.jl = NG; C.jr = NG + cfg->ny;
  C.kl = cfg->boost_invariant ? 0 : NG; C.kr = cfg->boost_invariant ? 1 : NG + cfg->nz;
  C.n = (long long)C.px * C.gy * C.gz;
  C.cart = cfg->coords == VH_COORD_CARTESIAN;
  C.bi = cfg->boost_invariant != 0;
  C.recon = cfg->recon;
  C.mirror = cfg->gubser_mirror != 0;
  C.dx = cfg->dx; C.dy = cfg->dy; C.dz = cfg->boost_invariant ? 1.0 : cfg->dz;
  C.eos_kind = cfg->eos_kind; C.eos_a = cfg->eos_a; C.eos_n = 0;
  C.etas0 = cfg->etas0; C.etas1 = cfg->etas1; C.etas_tc = cfg->etas_tc; C.hbarc = cfg->hbarc;
  C.taupi_kind = cfg->taupi_kind;
  C.taupi_c = cfg->taupi_const;
  C.cold = cfg->cold_plasma != 0;
  C.mm_theta = cfg->minmod_theta;
  h->tau = cfg->tau0;
  if (const char* v = std::getenv("VH_PDL")) h->pdl = std::strcmp(v, "0") != 0;
  if (const char* v = std::getenv("VH_TMA")) h->tma_wanted = std::strcmp(v, "0") != 0;

  auto bail = [&](cudaError_t e, const char* what) {
    g_create_err = std::string("vh_create: ") + what + ": " + cudaGetErrorString(e);
    vh_destroy(h);
    return e == cudaErrorMemoryAllocation ? VH_E_NOMEM : VH_E_CUDA;
  };
  cudaError_t e;
  if (cfg->eos_kind == VH_EOS_TABLE) {
    const int n = cfg->eos_n;
    std::vector<double> t(4 * (size_t)n);
    std::vector<float> tf(4 * (size_t)n);
    for (int i = 0; i < n; i++) {
      t[i] = cfg->eos_e[i]; t[n + i] = cfg->eos_p[i]; t[2 * n + i] = cfg->eos_cs2[i]; t[3 * n + i] = cfg->eos_t[i];
    }
    for (size_t i = 0; i < t.size(); i++) tf[i] = (float)t[i];
    h->eos_host = t;
    if ((e = cudaMalloc(&h->eos_d, sizeof(double) * t.size())) != cudaSuccess) return bail(e, "eos table");
    if ((e = cudaMalloc(&h->eos_f, sizeof(float) * t.size())) != cudaSuccess) return bail(e, "eos table");
    if ((e = cudaMemcpy(h->eos_d, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
      return bail(e, "eos table");
    if ((e = cudaMemcpy(h->eos_f, tf.data(), sizeof(float) * t.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
      return bail(e, "eos table");
    C.eos_n = n;
    C.eos_l0 = std::log(cfg->eos_e[0]);
    C.eos_idl = (n - 1) / (std::log(cfg->eos_e[n - 1]) - C.eos_l0);
    C.eos_d = h->eos_d;
    C.eos_f = h->eos_f;
  }
  const size_t bytes = (size_t)kStateArrays * C.n * h->esz;
  if ((e = cudaMalloc(&h->state, bytes)) != cudaSuccess) return bail(e, "state");
  if ((e = cudaMemset(h->state, 0, bytes)) != cudaSuccess) return bail(e, "state");
  if ((e = cudaMalloc(&h->stage, sizeof(double) * 18 * C.n)) != cudaSuccess) return bail(e, "staging");
  if ((e = cudaMalloc(&h->status, sizeof(unsigned int))) != cudaSuccess) return bail(e, "status");
  if ((e = cudaMalloc(&h->iters, sizeof(unsigned long long))) != cudaSuccess) return bail(e, "iters");
  if ((e = cudaMalloc(&h->red, sizeof(unsigned long long) * 4)) != cudaSuccess) return bail(e, "reduce");
  h->part_blocks = 296;
  if ((e = cudaMalloc(&h->part, sizeof(double) * 8 * h->part_blocks + 32)) != cudaSuccess) return bail(e, "reduce");
  if ((e = cudaMemset(h->status, 0, sizeof(unsigned int))) != cudaSuccess) return bail(e, "status");
  if ((e = cudaMemset(h->iters, 0, sizeof(unsigned long long))) != cudaSuccess) return bail(e, "iters");
  set_ptrs(h->pd, h->state, C.n, h->status, h->iters);
  set_ptrs(h->pf, h->state, C.n, h->status, h->iters);
  if ((h->mixed ? set_smem_attrs<float>(h) : set_smem_attrs<double>(h)) != VH_OK) {
    g_create_err = "vh_create: " + h->err;
    vh_destroy(h);
    return VH_E_CUDA;
  }
  *out = h;
  return VH_OK;
}

extern "C" int vh_destroy(vh_handle* h) {
  if (!h) return VH_OK;
  cudaFree(h->state); cudaFree(h->stage); cudaFree(h->eos_d); cudaFree(h->eos_f);
  cudaFree(h->status); cudaFree(h->iters); cudaFree(h->red); cudaFree(h->part);
  cudaFree(h->adj_buf); cudaFree(h->fo_prev); cudaFree(h->xfer);
  delete h;
  return VH_OK;
}

extern "C" int vh_set_stream(vh_handle* h, void* stream) {
  if (!h) return VH_E_ARG;
  h->stream = static_cast<cudaStream_t>(stream);
  return VH_OK;
}

extern "C" int vh_dims(const vh_handle* h, int* gx, int* gy, int* gz) {
  if (!h || !gx || !gy || !gz) return VH_E_ARG;
  *gx = h->C.gx; *gy = h->C.gy; *gz = h->C.gz;
  return VH_OK;
}


// canonical doubles (18 fields; host or device) -> state
static int import_state(vh_handle* h, const double* canon) {
  const long long n18 = 18 * h->C.n;
  if (h->mixed) {
    if (int r = pitched_in(h, h->stage, canon, 18)) return r;
    k_d2f<<<grid1(n18, 256), 256, 0, h->stream>>>(h->stage, static_cast<float*>(h->state), n18);
  } else if (canon != h->state) {
    if (int r = pitched_in(h, static_cast<double*>(h->state), canon, 18)) return r;
  }
  VH_CUDA(h, cudaGetLastError());
  return VH_OK;
}
static int export_state(vh_handle* h, double* canon) {
  const long long n18 = 18 * h->C.n;
  if (h->mixed) {
    k_f2d<<<grid1(n18, 256), 256, 0, h->stream>>>(static_cast<const float*>(h->state), h->stage, n18);
    VH_CUDA(h, cudaGetLastError());
    return pitched_out(h, canon, h->stage, 18);
  }
  return pitched_out(h, canon, static_cast<const double*>(h->state), 18);
}

static int state_was_set(vh_handle* h, double tau) {
  h->tau = tau;
  h->have_state = true;
  h->fo_have = false;
  VH_CUDA(h, cudaMemsetAsync(h->status, 0, sizeof(unsigned int), h->stream));
  return VH_OK;
}
extern "C" int vh_set_state_device(vh_handle* h, const double* dev, double tau) {
  if (!h || !dev) return VH_E_ARG;
  if (int r = import_state(h, dev)) return r;
  return state_was_set(h, tau);
}
extern "C" int vh_get_state_device(vh_handle* h, double* dev) {
  if (!h || !dev) return VH_E_ARG;
  if (!h->have_state) return fail(h, VH_E_STATE, "no state set");
  return export_state(h, dev);
}
extern "C" int vh_set_state(vh_handle* h, const double* host, double tau) {
  if (!h || !host) return VH_E_ARG;
  if (int r = import_state(h, host)) return r;
  return state_was_set(h, tau);
}
extern "C" int vh_get_state(vh_handle* h, double* host) {
  if (!h || !host) return VH_E_ARG;
  if (!h->have_state) return fail(h, VH_E_STATE, "no state set");
  if (int r = export_state(h, host)) return r;
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  return VH_OK;
}


extern "C" int vh_step(vh_handle* h, int nsteps) {
  if (!h || nsteps < 0) return VH_E_ARG;
  if (!h->have_state) return fail(h, VH_E_STATE, "vh_step before vh_set_state / vh_init_profile");
  VH_CUDA(h, cudaMemsetAsync(h->iters, 0, sizeof(unsigned long long), h->stream));
  for (int s = 0; s < nsteps; s++) {
    int r = h->mixed ? step_once<float>(h, h->pf) : step_once<double>(h, h->pd);
    if (r) return r;
  }
  return read_status(h);
}

// Steps with a CUDA event pair around every launch, accumulating device
// milliseconds per kernel kind: out[0..2] k_dir x/y/eta, out[3] k_update
// stage 1, out[4] k_update stage 2 (summed over nsteps steps).
template <class R>
static int timed_steps(vh_handle* h, const DevPtrs<R>& P, int nsteps, double* out) {
  const DevCfg& C = h->C;
  cudaEvent_t ev[2];
  VH_CUDA(h, cudaEventCreate(&ev[0]));
  VH_CUDA(h, cudaEventCreate(&ev[1]));
  for (int q = 0; q < 5; q++) out[q] = 0;
  auto timed = [&](int slot, auto&& launch) -> int {
    VH_CUDA(h, cudaEventRecord(ev[0], h->stream));
    int r = launch();
    if (r) return r;
    VH_CUDA(h, cudaEventRecord(ev[1], h->stream));
    VH_CUDA(h, cudaEventSynchronize(ev[1]));
    float ms = 0;
    VH_CUDA(h, cudaEventElapsedTime(&ms, ev[0], ev[1]));
    out[slot] += ms;
    return VH_OK;
  };
  int r = VH_OK;
  for (int s = 0; s < nsteps && !r; s++) {
    const double tau = h->tau, ts = h->cfg.dtau;
    for (int stage = 0; stage < 2 && !r; stage++) {
      const double t = stage ? tau + ts : tau;
      for (int d = 0; d < (C.bi ? 2 : 3) && !r; d++)
        r = timed(d, [&]() { return launch_dir<R>(h, P, d, stage, t, d == 0); });
      if (r) break;
      r = timed(3 + stage, [&]() -> int {
        return stage == 0 ? stage_update<R, 1>(h, P, tau, ts) : stage_update<R, 2>(h, P, tau, ts);
      });
    }
    h->tau = tau + ts;
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  return r;
}

extern "C" int vh_time_kernels(vh_handle* h, int nsteps, double* ms_out) {
  if (!h || !ms_out || nsteps < 0) return VH_E_ARG;
  if (!h->have_state) return fail(h, VH_E_STATE, "no state set");
  int r = h->mixed ? timed_steps<float>(h, h->pf, nsteps, ms_out) : timed_steps<double>(h, h->pd, nsteps, ms_out);
  if (r) return r;
  return read_status(h);
}

extern "C" int vh_get_time(const vh_handle* h, double* tau) {
  if (!h || !tau) return VH_E_ARG;
  *tau = h->tau;
  return VH_OK;
}

extern "C" int vh_sweep_uses_tma(const vh_handle* h, int* tma) {
  if (!h || !tma) return VH_E_ARG;
  *tma = h->tma ? 1 : 0;
  return VH_OK;
}

extern "C" int vh_last_iterations(vh_handle* h, long long* iters) {
  if (!h || !iters) return VH_E_ARG;
  unsigned long long v = 0;
  VH_CUDA(h, cudaMemcpyAsync(&v, h->iters, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  *iters = (long long)v;
  return VH_OK;
}

template <class R>
static int init_tail(vh_handle* h, const DevPtrs<R>& P, int pi_mode, double tau) {
  const DevCfg& C = h->C;
  if (pi_mode == VH_PI_NS) {
    R* du16 = reinterpret_cast<R*>(h->stage);  // 16*n fits in the 18*n staging buffer
    k_du_full<R><<<grid1(C.n, 128), 128, 0, h->stream>>>(C, P, du16, h->cfg.dtau);
    k_ns_pi<R><<<grid1(C.n, 128), 128, 0, h->stream>>>(C, P, du16, tau);
  }
  k_fill_tmunu<R><<<grid1(C.n, 256), 256, 0, h->stream>>>(C, P, tau);
  VH_CUDA(h, cudaGetLastError());
  return VH_OK;
}

extern "C" int vh_init_profile(vh_handle* h, double tau, const double* e, const double* ux, const double* uy,
                               const double* ueta, const double* prevu4, int pi_mode, const double* pi5) {
  if (!h || !e || !ux || !uy) return VH_E_ARG;
  if (pi_mode != VH_PI_GIVEN && pi_mode != VH_PI_ZERO && pi_mode != VH_PI_NS) return fail(h, VH_E_ARG, "pi_mode");
  if (pi_mode == VH_PI_GIVEN && !pi5) return fail(h, VH_E_ARG, "pi5 is required with VH_PI_GIVEN");
  const long long n = canon_cells(h->C);
  const double t2 = h->C.cart ? 1.0 : tau * tau;
  std::vector<double> f(18 * (size_t)n, 0.0);
  for (long long c = 0; c < n; c++) {
    const double ue = ueta ? ueta[c] : 0.0;
    f[c] = e[c];
    f[2 * n + c] = ux[c];
    f[3 * n + c] = uy[c];
    f[4 * n + c] = ue;
    f[1 * n + c] = std::sqrt(1 + ux[c] * ux[c] + uy[c] * uy[c] + t2 * ue * ue);
    for (int l = 0; l < 5; l++) f[(5 + l) * n + c] = (pi_mode == VH_PI_GIVEN) ? pi5[l * n + c] : 0.0;
    for (int l = 0; l < 4; l++) f[(14 + l) * n + c] = prevu4 ? prevu4[l * n + c] : f[(1 + l) * n + c];
  }
  int r = vh_set_state(h, f.data(), tau);
  if (r) return r;
  r = h->mixed ? init_tail<float>(h, h->pf, pi_mode, tau) : init_tail<double>(h, h->pd, pi_mode, tau);
  if (r) return r;
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  return VH_OK;
}

extern "C" int vh_get_primitive(vh_handle* h, double* e, double* P, double* T, double* u4, double* pi10) {
  if (!h) return VH_E_ARG;
  if (!h->have_state) return fail(h, VH_E_STATE, "no state set");
  const long long n = h->C.n;
  double* buf = h->stage;  // 18 x n doubles; 17 are used
  if (h->mixed) k_primitive<float><<<grid1(n, 256), 256, 0, h->stream>>>(h->C, h->pf, h->tau, buf);
  else k_primitive<double><<<grid1(n, 256), 256, 0, h->stream>>>(h->C, h->pd, h->tau, buf);
  VH_CUDA(h, cudaGetLastError());
  int r = VH_OK;
  if (e && !r) r = pitched_out(h, e, buf, 1);
  if (P && !r) r = pitched_out(h, P, buf + n, 1);
  if (T && !r) r = pitched_out(h, T, buf + 2 * n, 1);
  if (u4 && !r) r = pitched_out(h, u4, buf + 3 * n, 4);
  if (pi10 && !r) r = pitched_out(h, pi10, buf + 7 * n, 10);
  if (r) return r;
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  return VH_OK;
}

extern "C" int vh_freezeout_step(vh_handle* h, double t_fo, double* out, long long cap, long long* count) {
  if (!h || !count || cap < 0 || (cap > 0 && !out) || !(t_fo > 0)) return VH_E_ARG;
  if (!h->have_state) return fail(h, VH_E_STATE, "no state set");
  const vh_config& c = h->cfg;
  if (h->C.cart) return fail(h, VH_E_UNSUPPORTED, "freeze-out surfaces are built on Milne grids");
  if (c.nx < 2 || c.ny < 2 || (!c.boost_invariant && c.nz < 2))
    return fail(h, VH_E_ARG, "a freeze-out surface needs two cells along every axis");
  const long long n = h->C.n, nc = canon_cells(h->C);
  const size_t nb = sizeof(double) * (size_t)nc;
  // two canonical slices (5 fields each): the kept one and the current one
  if (!h->fo_prev) VH_CUDA(h, cudaMalloc(&h->fo_prev, 10 * nb));
  // T and u^mu of the current state: rows 2 (T) and 3..6 (u^mu) of the
  // primitive fields, contiguous, in the canonical layout the surface
  // kernels read
  double* buf = h->stage;
  if (h->mixed) k_primitive<float><<<grid1(n, 256), 256, 0, h->stream>>>(h->C, h->pf, h->tau, buf);
  else k_primitive<double><<<grid1(n, 256), 256, 0, h->stream>>>(h->C, h->pd, h->tau, buf);
  VH_CUDA(h, cudaGetLastError());
  double* cur = h->fo_prev + 5 * nc;
  if (int r = pitched_out(h, cur, buf + 2 * n, 5)) return r;
  *count = 0;
  if (h->fo_have) {
    if (!(h->tau > h->fo_tau)) return fail(h, VH_E_STATE, "no step since the last freeze-out slice");
    const double* prev = h->fo_prev;
    const int r = c.boost_invariant
                      ? vh_freezeout_2d_device(c.nx, c.ny, c.dx, c.dy, h->fo_tau, h->tau, prev, cur, prev + nc,
                                               cur + nc, t_fo, out, cap, count, h->stream)
                      : vh_freezeout_3d_device(c.nx, c.ny, c.nz, c.dx, c.dy, c.dz, h->fo_tau, h->tau, prev, cur,
                                               prev + nc, cur + nc, t_fo, out, cap, count, h->stream);
    if (r == VH_E_ARG && *count > cap)
      return fail(h, VH_E_ARG, "the surface has " + std::to_string(*count) + " elements, more than cap; the slice "
                               "is kept for a call with room for them");
    if (r) return fail(h, r, "freeze-out surface between two slices");
  }
  VH_CUDA(h, cudaMemcpyAsync(h->fo_prev, cur, 5 * nb, cudaMemcpyDeviceToDevice, h->stream));
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  h->fo_tau = h->tau;
  h->fo_have = true;
  return VH_OK;
}

template <class R>
static int ns_pi10(vh_handle* h, const DevPtrs<R>& P, double* out) {
  const DevCfg& C = h->C;
  R* du16 = P.base1;  // 16 of the step's 34 scratch arrays, free between steps
  k_du_full<R><<<grid1(C.n, 128), 128, 0, h->stream>>>(C, P, du16, h->cfg.dtau);
  k_ns_pi10<R><<<grid1(C.n, 128), 128, 0, h->stream>>>(C, P, du16, h->tau, out);
  VH_CUDA(h, cudaGetLastError());
  return VH_OK;
}

extern "C" int vh_get_conserved(vh_handle* h, double* var10) {
  if (!h || !var10) return VH_E_ARG;
  if (!h->have_state) return fail(h, VH_E_STATE, "no state set");
  const size_t n = (size_t)canon_cells(h->C);
  std::vector<double> f(18 * n);
  int r = vh_get_state(h, f.data());
  if (r) return r;
  // NEWEST5/hydroKT.h:345-361 (TXYZ5/hydroKT.h:270-286 without the tau)
  const double t = h->C.cart ? 1.0 : h->tau;
  for (int l = 0; l < 4; l++)
    for (size_t c = 0; c < n; c++) var10[l * n + c] = t * f[(10 + l) * n + c];
  for (int l = 0; l < 5; l++) std::copy(f.begin() + (5 + l) * n, f.begin() + (6 + l) * n, var10 + (4 + l) * n);
  std::fill(var10 + 9 * n, var10 + 10 * n, 0.0);  // bulk pressure: not evolved
  return VH_OK;
}

extern "C" int vh_get_ns_pi(vh_handle* h, double* pi10) {
  if (!h || !pi10) return VH_E_ARG;
  if (!h->have_state) return fail(h, VH_E_STATE, "no state set");
  const long long n = h->C.n;
  double* buf = h->stage;  // 18 x n doubles; 10 are used
  int r = h->mixed ? ns_pi10<float>(h, h->pf, buf) : ns_pi10<double>(h, h->pd, buf);
  if (r) return r;
  (void)n;
  if ((r = pitched_out(h, pi10, buf, 10))) return r;
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  return VH_OK;
}

extern "C" int vh_landau_match(const double* tmunu10, long long n, double tau, int cartesian, double* e, double* u4,
                               long long* nfail) {
  if (!tmunu10 || !e || !u4 || n < 1 || (!cartesian && !(tau > 0))) return VH_E_ARG;
  double* d = nullptr;
  unsigned long long* cnt = nullptr;
  const size_t nb = sizeof(double) * (size_t)n;
  if (cudaMalloc(&d, 15 * nb) != cudaSuccess) {
    g_create_err = "vh_landau_match: device buffers";
    return VH_E_NOMEM;
  }
  if (cudaMalloc(&cnt, sizeof(unsigned long long)) != cudaSuccess) {
    cudaFree(d);
    g_create_err = "vh_landau_match: device buffers";
    return VH_E_NOMEM;
  }
  unsigned long long bad = 0;
  cudaError_t err = cudaMemcpy(d, tmunu10, 10 * nb, cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaMemset(cnt, 0, sizeof(bad));
  if (err == cudaSuccess) {
    k_landau<double><<<grid1(n, 128), 128>>>(n, tau, cartesian, d, d + 10 * n, d + 11 * n, cnt);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) err = cudaMemcpy(e, d + 10 * n, nb, cudaMemcpyDeviceToHost);
  if (err == cudaSuccess) err = cudaMemcpy(u4, d + 11 * n, 4 * nb, cudaMemcpyDeviceToHost);
  if (err == cudaSuccess) err = cudaMemcpy(&bad, cnt, sizeof(bad), cudaMemcpyDeviceToHost);
  cudaFree(d);
  cudaFree(cnt);
  if (err != cudaSuccess) {
    g_create_err = std::string("vh_landau_match: ") + cudaGetErrorString(err);
    return VH_E_CUDA;
  }
  if (nfail) *nfail = (long long)bad;
  return VH_OK;
}

extern "C" int vh_init_tmunu(vh_handle* h, double tau, const double* tmunu10, long long* nfail) {
  if (!h || !tmunu10) return VH_E_ARG;
  if (!h->C.cart && !(tau > 0)) return fail(h, VH_E_ARG, "Milne tau must be positive");
  const long long n = h->C.n;
  double* buf = h->stage;  // 18 x n doubles; the tensor takes 10
  if (int r = pitched_in(h, buf, tmunu10, 10)) return r;
  VH_CUDA(h, cudaMemsetAsync(h->red, 0, sizeof(unsigned long long), h->stream));
  if (h->mixed) {
    k_init_tmunu<float><<<grid1(n, 128), 128, 0, h->stream>>>(h->C, h->pf, tau, buf, h->red);
    k_fill_tmunu<float><<<grid1(n, 256), 256, 0, h->stream>>>(h->C, h->pf, tau);
  } else {
    k_init_tmunu<double><<<grid1(n, 128), 128, 0, h->stream>>>(h->C, h->pd, tau, buf, h->red);
    k_fill_tmunu<double><<<grid1(n, 256), 256, 0, h->stream>>>(h->C, h->pd, tau);
  }
  VH_CUDA(h, cudaGetLastError());
  unsigned long long bad = 0;
  VH_CUDA(h, cudaMemcpyAsync(&bad, h->red, sizeof(bad), cudaMemcpyDeviceToHost, h->stream));
  VH_CUDA(h, cudaMemsetAsync(h->status, 0, sizeof(unsigned int), h->stream));
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  h->tau = tau;
  h->have_state = true;
  h->fo_have = false;
  if (nfail) *nfail = (long long)bad;
  if (bad) return fail(h, VH_E_ROOTFIND, "Landau matching found no timelike eigenvector in " + std::to_string(bad) +
                                             " cell(s)");
  return VH_OK;
}

extern "C" int vh_init_prevu_tmunu(vh_handle* h, double tau_prev, const double* tmunu10, long long* nfail) {
  if (!h || !tmunu10) return VH_E_ARG;
  if (!h->have_state) return fail(h, VH_E_STATE, "vh_init_prevu_tmunu after the state is set");
  if (!h->C.cart && !(tau_prev > 0)) return fail(h, VH_E_ARG, "Milne tau must be positive");
  const long long n = h->C.n;
  double* buf = h->stage;
  if (int r = pitched_in(h, buf, tmunu10, 10)) return r;
  VH_CUDA(h, cudaMemsetAsync(h->red, 0, sizeof(unsigned long long), h->stream));
  if (h->mixed) k_prevu_tmunu<float><<<grid1(n, 128), 128, 0, h->stream>>>(h->C, h->pf, tau_prev, buf, h->red);
  else k_prevu_tmunu<double><<<grid1(n, 128), 128, 0, h->stream>>>(h->C, h->pd, tau_prev, buf, h->red);
  VH_CUDA(h, cudaGetLastError());
  unsigned long long bad = 0;
  VH_CUDA(h, cudaMemcpyAsync(&bad, h->red, sizeof(bad), cudaMemcpyDeviceToHost, h->stream));
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  if (nfail) *nfail = (long long)bad;
  if (bad) return fail(h, VH_E_ROOTFIND, "Landau matching found no timelike eigenvector in " + std::to_string(bad) +
                                             " cell(s)");
  return VH_OK;
}

extern "C" int vh_max_temperature(vh_handle* h, double* tmax_gev) {
  if (!h || !tmax_gev) return VH_E_ARG;
  if (!h->have_state) return fail(h, VH_E_STATE, "no state set");
  VH_CUDA(h, cudaMemsetAsync(h->red, 0, sizeof(unsigned long long), h->stream));
  if (h->mixed) k_max_temp<float><<<296, 256, 0, h->stream>>>(h->C, h->pf, h->red);
  else k_max_temp<double><<<296, 256, 0, h->stream>>>(h->C, h->pd, h->red);
  VH_CUDA(h, cudaGetLastError());
  unsigned long long bits = 0;
  VH_CUDA(h, cudaMemcpyAsync(&bits, h->red, sizeof(bits), cudaMemcpyDeviceToHost, h->stream));
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  std::memcpy(tmax_gev, &bits, sizeof(double));
  return VH_OK;
}

extern "C" int vh_conservation_sums(vh_handle* h, double* out4) {
  if (!h || !out4) return VH_E_ARG;
  if (!h->have_state) return fail(h, VH_E_STATE, "no state set");
  const double dv = h->C.dx * h->C.dy * (h->C.bi ? 1.0 : h->C.dz);
  double* fin = h->part + 8 * h->part_blocks;
  if (h->mixed) k_conserve_part<float><<<h->part_blocks, 256, 0, h->stream>>>(h->C, h->pf, h->tau, dv, h->part);
  else k_conserve_part<double><<<h->part_blocks, 256, 0, h->stream>>>(h->C, h->pd, h->tau, dv, h->part);
  k_conserve_final<<<1, 32, 0, h->stream>>>(h->part, h->part_blocks, fin);
  VH_CUDA(h, cudaGetLastError());
  VH_CUDA(h, cudaMemcpyAsync(out4, fin, sizeof(double) * 4, cudaMemcpyDeviceToHost, h->stream));
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  return VH_OK;
}

extern "C" int vh_cfl(vh_handle* h, double* max_speed, double* dtau_suggest) {
  if (!h || !max_speed || !dtau_suggest) return VH_E_ARG;
  if (!h->have_state) return fail(h, VH_E_STATE, "no state set");
  VH_CUDA(h, cudaMemsetAsync(h->red, 0, sizeof(unsigned long long), h->stream));
  if (h->mixed) k_cfl<float><<<296, 256, 0, h->stream>>>(h->C, h->pf, h->tau, h->red);
  else k_cfl<double><<<296, 256, 0, h->stream>>>(h->C, h->pd, h->tau, h->red);
  VH_CUDA(h, cudaGetLastError());
  unsigned long long bits = 0;
  VH_CUDA(h, cudaMemcpyAsync(&bits, h->red, sizeof(bits), cudaMemcpyDeviceToHost, h->stream));
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  std::memcpy(max_speed, &bits, sizeof(double));
  *dtau_suggest = *max_speed > 0 ? h->C.dx / (8.0 * *max_speed) : INFINITY;
  return VH_OK;
}

template <class R>
static int debug_terms(vh_handle* h, const DevPtrs<R>& P, double* res, double* src, double* du) {
  const DevCfg& C = h->C;
  const long long n = C.n;
  int r;
  if ((r = stage_rhs<R>(h, P, 0, h->tau))) return r;
  R* du16 = reinterpret_cast<R*>(h->stage);
  k_du_full<R><<<grid1(n, 128), 128, 0, h->stream>>>(C, P, du16, h->cfg.dtau);
  // the spatial derivatives along each direction come from k_dir (interior)
  R* src9 = nullptr;
  VH_CUDA(h, cudaMallocAsync(&src9, sizeof(R) * 9 * n, h->stream));
  k_debug_src<R><<<grid1(n, 128), 128, 0, h->stream>>>(C, P, du16, src9, h->tau);
  VH_CUDA(h, cudaGetLastError());
  std::vector<R> tmp(16 * (size_t)n);
  // device fields (rows of px cells) -> canonical doubles (rows of gx)
  const long long nc = canon_cells(C), rows = (long long)C.gy * C.gz;
  auto unpad = [&](double* dst, int nf) {
    for (int q = 0; q < nf; q++)
      for (long long r = 0; r < rows; r++)
        for (int i = 0; i < C.gx; i++) dst[q * nc + r * C.gx + i] = (double)tmp[q * n + r * C.px + i];
  };
  VH_CUDA(h, cudaMemcpyAsync(tmp.data(), P.res(0), sizeof(R) * 9 * n, cudaMemcpyDeviceToHost, h->stream));
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  unpad(res, 9);
  VH_CUDA(h, cudaMemcpyAsync(tmp.data(), src9, sizeof(R) * 9 * n, cudaMemcpyDeviceToHost, h->stream));
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  unpad(src, 9);
  VH_CUDA(h, cudaMemcpyAsync(tmp.data(), du16, sizeof(R) * 16 * n, cudaMemcpyDeviceToHost, h->stream));
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  unpad(du, 16);
  VH_CUDA(h, cudaFreeAsync(src9, h->stream));
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  return VH_OK;
}

extern "C" int vh_debug_stage_terms(vh_handle* h, double* res, double* src, double* du) {
  if (!h || !res || !src || !du) return VH_E_ARG;
  if (!h->have_state) return fail(h, VH_E_STATE, "no state set");
  return h->mixed ? debug_terms<float>(h, h->pf, res, src, du) : debug_terms<double>(h, h->pd, res, src, du);
}

extern "C" const char* vh_last_error(const vh_handle* h) {
  return h ? h->err.c_str() : g_create_err.c_str();
}

int vh_internal_error(vh_handle* h, int code, const char* msg) { return fail(h, code, msg); }

int vh_internal_config(const vh_handle* h, vh_config* out, std::vector<double>* eos4) {
  if (!h || !out) return VH_E_ARG;
  *out = h->cfg;
  if (eos4) *eos4 = h->eos_host;
  return VH_OK;
}
