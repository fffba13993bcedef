// Batched ensemble of boost-invariant events: one pool of device state for
// all events, a packed event table, and one persistent kernel that advances
// every live event through whole TVDRK2 steps (flux sweeps, update) with
// grid-wide barriers between the phases.  Each event has its own tau, dtau
// and stopping rule (maximum temperature below t_freeze, or tau_max), the
// reference's main-loop break (NEWEST5/main.cpp:188-205) applied per event.
// Launches are recorded into a CUDA graph and replayed; tile shape, occupancy,
// unroll and steps per launch come from an autotuner (vh_batch_autotune).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "vh.h"
#include "vh_adjoint.cuh"
#include "vh_aux.cuh"
#include "vh_nvtx.h"

using namespace vh;

namespace {

enum : int { EV_RUNNING = 0, EV_FROZEN = 1, EV_TAUMAX = 2, EV_FAILED = 3 };

struct Tables {
  int n_events;
  const long long* off;
  const int* nx;
  const int* ny;
  double* tau;
  const double* dtau;
  const double* tau_max;
  int* state;
  int* steps;
  unsigned long long* tmax_bits;
  unsigned int* flag;      // per-event failure bits (the event's DevPtrs status)
  const int4* xitems;      // {event, tile along x, tile across}
  int n_x;
  const int4* yitems;      // {event, tile along y, tile across}
  int n_y;
  const int2* uitems;      // {event, chunk of blockDim cells}
  int n_u;
  unsigned int* bar;       // [0] arrivals, [1] generation, [2] timeout flag
  int* running;            // events still running after the last launch
  unsigned long long* iters;
  double t_freeze_gev;
};

template <class R>
struct Args {
  DevCfg C0;
  DevPtrs<R> pool;
  Tables T;
};

__device__ inline DevCfg event_cfg(const DevCfg& C0, int nx, int ny) {
  DevCfg C = C0;
  C.nx = nx; C.ny = ny; C.nz = 1;
  C.gx = nx + 2 * NG; C.gy = ny + 2 * NG; C.gz = 1;
  C.px = C.gx;  // the pool keeps unpadded rows
  C.xt0 = NG;
  C.il = NG; C.ir = NG + nx; C.jl = NG; C.jr = NG + ny; C.kl = 0; C.kr = 1;
  C.n = (long long)C.gx * C.gy;
  return C;
}

// Grid-wide barrier among the co-resident blocks of a cooperative launch.
// The wait is bounded: after ~2 s the block sets the timeout flag and
// returns false, and every block leaves the kernel at its next check.
__device__ inline bool grid_barrier(unsigned int* bar, long long max_spins = 1ll << 24) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* vgen = bar + 1;
    const unsigned int g = *vgen;
    __threadfence();
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long spins = 0;
      while (*vgen == g) {
        if (++spins > max_spins) { atomicOr(bar + 2, 1u); break; }
        __nanosleep(128);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile unsigned int*)(bar + 2) == 0;
}

template <class R, int NC, int MINB, int UNR>
__global__ void __launch_bounds__(NC * 32, MINB) k_batch(Args<R> A, int nsteps) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  using SX = DirSmem<R, 0, NC>;
  using SY = DirSmem<R, 1, NC>;
  const Tables& T = A.T;
  __shared__ double red[32];
  for (int s = 0; s < nsteps; s++) {
    for (int stage = 0; stage < 2; stage++) {
      // ---- flux sweep along x, then y
      for (int it = blockIdx.x; it < T.n_x; it += gridDim.x) {
        const int4 w = T.xitems[it];
        const int ev = w.x;
        if (T.state[ev] != EV_RUNNING || T.flag[ev]) continue;
        const DevCfg C = event_cfg(A.C0, T.nx[ev], T.ny[ev]);
        DevPtrs<R> P = A.pool.shifted(T.off[ev]);
        P.status = T.flag + ev;
        const double tau = stage ? T.tau[ev] + T.dtau[ev] : T.tau[ev];
        dir_tile<R, 0, NC, UNR>(C, P, stage, (R)tau, (R)(1.0 / C.dx), (R)C.dx, 1, w.y, w.z, 0,
                                *reinterpret_cast<SX*>(smem_raw));
        __syncthreads();
      }
      if (!grid_barrier(T.bar)) return;
      for (int it = blockIdx.x; it < T.n_y; it += gridDim.x) {
        const int4 w = T.yitems[it];
        const int ev = w.x;
        if (T.state[ev] != EV_RUNNING || T.flag[ev]) continue;
        const DevCfg C = event_cfg(A.C0, T.nx[ev], T.ny[ev]);
        DevPtrs<R> P = A.pool.shifted(T.off[ev]);
        P.status = T.flag + ev;
        const double tau = stage ? T.tau[ev] + T.dtau[ev] : T.tau[ev];
        dir_tile<R, 1, NC, UNR>(C, P, stage, (R)tau, (R)(1.0 / C.dy), (R)C.dy, 0, w.y, w.z, 0,
                                *reinterpret_cast<SY*>(smem_raw));
        __syncthreads();
      }
      if (!grid_barrier(T.bar)) return;
      // ---- update: sources, RK, root-find, ghosts; stage 2 also reduces max T
      unsigned long long my_it = 0;
      for (int it = blockIdx.x; it < T.n_u; it += gridDim.x) {
        const int2 w = T.uitems[it];
        const int ev = w.x;
        if (T.state[ev] != EV_RUNNING || T.flag[ev]) continue;
        const DevCfg C = event_cfg(A.C0, T.nx[ev], T.ny[ev]);
        DevPtrs<R> P = A.pool.shifted(T.off[ev]);
        P.status = T.flag + ev;
        const long long t = (long long)w.y * blockDim.x + threadIdx.x;
        double tg = 0.0;
        if (t < (long long)C.nx * C.ny) {
          my_it += stage == 0 ? update_cell<R, 1>(C, P, T.tau[ev], T.dtau[ev], t, nullptr)
                              : update_cell<R, 2>(C, P, T.tau[ev], T.dtau[ev], t, &tg);
        }
        if (stage == 1) {
          for (int o = 16; o > 0; o >>= 1) tg = fmax(tg, __shfl_down_sync(0xffffffffu, tg, o));
          if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = tg;
          __syncthreads();
          if (threadIdx.x == 0) {
            double m = 0;
            for (int q = 0; q < (int)(blockDim.x >> 5); q++) m = fmax(m, red[q]);
            atomicMax(T.tmax_bits + ev, (unsigned long long)__double_as_longlong(m));
          }
          __syncthreads();
        }
      }
      for (int o = 16; o > 0; o >>= 1) my_it += __shfl_down_sync(0xffffffffu, my_it, o);
      if ((threadIdx.x & 31) == 0 && my_it) atomicAdd(T.iters, my_it);
      if (!grid_barrier(T.bar)) return;
    }
    // ---- end of step: advance time, apply each event's stopping rule
    for (int ev = blockIdx.x * blockDim.x + threadIdx.x; ev < T.n_events; ev += gridDim.x * blockDim.x) {
      if (T.state[ev] != EV_RUNNING) continue;
      if (T.flag[ev]) { T.state[ev] = EV_FAILED; continue; }
      T.tau[ev] += T.dtau[ev];
      T.steps[ev] += 1;
      const double tm = __longlong_as_double((long long)T.tmax_bits[ev]);
      T.tmax_bits[ev] = 0;
      if (tm < T.t_freeze_gev) T.state[ev] = EV_FROZEN;
      else if (T.tau[ev] >= T.tau_max[ev] - 1e-9) T.state[ev] = EV_TAUMAX;
    }
    if (!grid_barrier(T.bar)) return;
  }
  if (blockIdx.x == 0) {
    int cnt = 0;
    for (int ev = threadIdx.x; ev < T.n_events; ev += blockDim.x) cnt += T.state[ev] == EV_RUNNING;
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    __shared__ int rc[32];
    if ((threadIdx.x & 31) == 0) rc[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int q = 0; q < (int)(blockDim.x >> 5); q++) tot += rc[q];
      *T.running = tot;
    }
  }
}

// Probe of the bounded barrier: two blocks, of which `absent` never arrive;
// block 0 waits at grid_barrier and, with a block missing, gives up after
// 2^20 polls (a fraction of a second) and sets the timeout flag.
__global__ void k_barrier_probe(unsigned int* bar, int absent) {
  if ((int)blockIdx.x >= (int)gridDim.x - absent) return;
  grid_barrier(bar, 1ll << 20);
}

// copy one event's canonical doubles (18 x n) into its pool view
template <class R>
__global__ void k_import_event(const double* src, DevPtrs<R> P, long long n) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  for (int q = 0; q < 18; q++) P.f(q)[c] = (R)src[q * n + c];
}
template <class R>
__global__ void k_export_event(DevPtrs<R> P, double* dst, long long n) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  for (int q = 0; q < 18; q++) dst[q * n + c] = (double)P.f(q)[c];
}

// one compiled configuration of the persistent kernel
struct Variant {
  int nc, minb, unr;
};
const Variant kVariants[] = {{4, 4, 1}, {4, 3, 1}, {8, 2, 1}, {8, 2, 3}, {8, 1, 1}};
constexpr int kNumVariants = 5;
const int kStepsChoices[] = {8, 32};

}  // namespace

struct vh_batch {
  vh_config cfg{};
  DevCfg C0{};
  bool mixed = false;
  size_t esz = 8;
  int n = 0;
  long long ntot = 0;
  std::vector<long long> off;
  std::vector<int> nx, ny;
  std::vector<double> tau0, dtau, tau_max;
  void* pool = nullptr;
  double* eos_d = nullptr;
  float* eos_f = nullptr;
  // device tables
  long long* d_off = nullptr;
  int *d_nx = nullptr, *d_ny = nullptr, *d_state = nullptr, *d_steps = nullptr, *d_running = nullptr;
  double *d_tau = nullptr, *d_dtau = nullptr, *d_taumax = nullptr;
  unsigned long long *d_tmax = nullptr, *d_iters = nullptr;
  unsigned int *d_flag = nullptr, *d_bar = nullptr;
  int4 *d_x[2] = {nullptr, nullptr}, *d_y[2] = {nullptr, nullptr};
  int n_xi[2] = {0, 0}, n_yi[2] = {0, 0};
  int2* d_u = nullptr;
  int n_ui = 0;
  double* stage = nullptr;  // staging for imports (18 x largest event)
  long long stage_cells = 0;
  double t_freeze_gev = 0.15;
  int variant = 2, steps_per_launch = 32, grid = 0;
  bool use_graph = true;
  std::string err;
};

static std::string g_batch_err;

#define VB_CUDA(b, call)                                                             \
  do {                                                                               \
    cudaError_t _e = (call);                                                         \
    if (_e != cudaSuccess) {                                                         \
      (b)->err = std::string(#call) + ": " + cudaGetErrorString(_e);                 \
      return VH_E_CUDA;                                                              \
    }                                                                                \
  } while (0)

template <class R>
static DevPtrs<R> pool_ptrs(vh_batch* b) {
  DevPtrs<R> P{};
  P.base0 = static_cast<R*>(b->pool);
  P.base1 = static_cast<R*>(b->pool) + 18 * b->ntot;
  P.stride = b->ntot;
  P.status = nullptr;
  P.iters = b->d_iters;
  return P;
}

static int build_items(vh_batch* b) {
  // x and y tiles for NC = 4 and 8 lines, update chunks of the block size
  for (int q = 0; q < 2; q++) {
    const int nc = q == 0 ? 4 : 8, tl = 26;
    std::vector<int4> xs, ys;
    for (int e = 0; e < b->n; e++) {
      for (int by = 0; by < (b->ny[e] + nc - 1) / nc; by++)
        for (int bx = 0; bx < (b->nx[e] + tl - 1) / tl; bx++) xs.push_back(make_int4(e, bx, by, 0));
      for (int bx = 0; bx < (b->nx[e] + nc - 1) / nc; bx++)
        for (int by = 0; by < (b->ny[e] + tl - 1) / tl; by++) ys.push_back(make_int4(e, by, bx, 0));
    }
    b->n_xi[q] = (int)xs.size();
    b->n_yi[q] = (int)ys.size();
    VB_CUDA(b, cudaMalloc(&b->d_x[q], sizeof(int4) * xs.size()));
    VB_CUDA(b, cudaMalloc(&b->d_y[q], sizeof(int4) * ys.size()));
    VB_CUDA(b, cudaMemcpy(b->d_x[q], xs.data(), sizeof(int4) * xs.size(), cudaMemcpyHostToDevice));
    VB_CUDA(b, cudaMemcpy(b->d_y[q], ys.data(), sizeof(int4) * ys.size(), cudaMemcpyHostToDevice));
  }
  return VH_OK;
}

static int build_uitems(vh_batch* b, int block) {
  std::vector<int2> us;
  for (int e = 0; e < b->n; e++) {
    const long long cells = (long long)b->nx[e] * b->ny[e];
    for (long long c = 0; c < (cells + block - 1) / block; c++) us.push_back(make_int2(e, (int)c));
  }
  if (b->d_u) cudaFree(b->d_u);
  b->n_ui = (int)us.size();
  VB_CUDA(b, cudaMalloc(&b->d_u, sizeof(int2) * us.size()));
  VB_CUDA(b, cudaMemcpy(b->d_u, us.data(), sizeof(int2) * us.size(), cudaMemcpyHostToDevice));
  return VH_OK;
}

extern "C" int vh_batch_create(const vh_config* cfg, int n_events, const int* nx, const int* ny, const double* tau0,
                               const double* dtau, const double* tau_max, double t_freeze_gev, vh_batch** out) {
  if (!cfg || !out || n_events < 1 || !nx || !ny || !tau0 || !dtau || !tau_max) return VH_E_ARG;
  *out = nullptr;
  if (!cfg->boost_invariant || cfg->coords != VH_COORD_MILNE) { g_batch_err = "batches hold boost-invariant Milne events"; return VH_E_UNSUPPORTED; }
  if (cfg->eos_kind == VH_EOS_TABLE && (cfg->eos_n < 2 || !cfg->eos_e)) return VH_E_ARG;
  vh_batch* b = new vh_batch();
  b->cfg = *cfg;
  b->mixed = cfg->precision == VH_PREC_MIXED;
  b->esz = b->mixed ? 4 : 8;
  b->n = n_events;
  long long tot = 0, big = 0;
  for (int e = 0; e < n_events; e++) {
    if (nx[e] < 3 || ny[e] < 3 || !(dtau[e] > 0) || !(tau0[e] > 0)) { delete b; return VH_E_ARG; }
    b->off.push_back(tot);
    const long long cells = (long long)(nx[e] + 6) * (ny[e] + 6);
    tot += cells;
    big = std::max(big, cells);
    b->nx.push_back(nx[e]); b->ny.push_back(ny[e]);
    b->tau0.push_back(tau0[e]); b->dtau.push_back(dtau[e]); b->tau_max.push_back(tau_max[e]);
  }
  b->ntot = tot;
  b->stage_cells = big;
  DevCfg& C = b->C0;
  C.nz = 1; C.gz = 1; C.kl = 0; C.kr = 1; C.cart = 0; C.bi = 1;
  C.recon = cfg->recon; C.mirror = cfg->gubser_mirror != 0;
  C.dx = cfg->dx; C.dy = cfg->dy; C.dz = 1.0;
  C.eos_kind = cfg->eos_kind; C.eos_a = cfg->eos_a;
  C.etas0 = cfg->etas0; C.etas1 = cfg->etas1; C.etas_tc = cfg->etas_tc; C.hbarc = cfg->hbarc;
  C.taupi_kind = cfg->taupi_kind; C.taupi_c = cfg->taupi_const; C.cold = cfg->cold_plasma != 0;
  C.mm_theta = cfg->minmod_theta;
  auto fail = [&](const char* what) {
    g_batch_err = std::string("vh_batch_create: ") + what + ": " + b->err;
    vh_batch_destroy(b);
    return VH_E_CUDA;
  };
  // a CUDA call's success, recording its error for fail()
  auto ok = [&](cudaError_t ce) {
    if (ce != cudaSuccess) b->err = cudaGetErrorString(ce);
    return ce == cudaSuccess;
  };
  if (cfg->eos_kind == VH_EOS_TABLE) {
    const int m = cfg->eos_n;
    std::vector<double> t(4 * (size_t)m);
    std::vector<float> tf(4 * (size_t)m);
    for (int i = 0; i < m; i++) { t[i] = cfg->eos_e[i]; t[m + i] = cfg->eos_p[i]; t[2 * m + i] = cfg->eos_cs2[i]; t[3 * m + i] = cfg->eos_t[i]; }
    for (size_t i = 0; i < t.size(); i++) tf[i] = (float)t[i];
    if (!ok(cudaMalloc(&b->eos_d, sizeof(double) * t.size())) || !ok(cudaMalloc(&b->eos_f, sizeof(float) * t.size())) ||
        !ok(cudaMemcpy(b->eos_d, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice)) ||
        !ok(cudaMemcpy(b->eos_f, tf.data(), sizeof(float) * t.size(), cudaMemcpyHostToDevice)))
      return fail("eos");
    C.eos_n = m; C.eos_l0 = std::log(cfg->eos_e[0]); C.eos_idl = (m - 1) / (std::log(cfg->eos_e[m - 1]) - C.eos_l0);
    C.eos_d = b->eos_d; C.eos_f = b->eos_f;
  }
  b->cfg.eos_e = b->cfg.eos_p = b->cfg.eos_cs2 = b->cfg.eos_t = nullptr;
  const size_t pool_bytes = (size_t)52 * tot * b->esz;
  cudaError_t ce = cudaMalloc(&b->pool, pool_bytes);
  if (ce != cudaSuccess) { b->err = cudaGetErrorString(ce); g_batch_err = "vh_batch_create: pool: " + b->err; vh_batch_destroy(b); return VH_E_NOMEM; }
  if (!ok(cudaMemset(b->pool, 0, pool_bytes))) return fail("pool");
  const int n = n_events;
  if (!ok(cudaMalloc(&b->d_off, sizeof(long long) * n)) || !ok(cudaMalloc(&b->d_nx, sizeof(int) * n)) ||
      !ok(cudaMalloc(&b->d_ny, sizeof(int) * n)) || !ok(cudaMalloc(&b->d_state, sizeof(int) * n)) ||
      !ok(cudaMalloc(&b->d_steps, sizeof(int) * n)) || !ok(cudaMalloc(&b->d_running, sizeof(int))) ||
      !ok(cudaMalloc(&b->d_tau, sizeof(double) * n)) || !ok(cudaMalloc(&b->d_dtau, sizeof(double) * n)) ||
      !ok(cudaMalloc(&b->d_taumax, sizeof(double) * n)) ||
      !ok(cudaMalloc(&b->d_tmax, sizeof(unsigned long long) * n)) ||
      !ok(cudaMalloc(&b->d_iters, sizeof(unsigned long long))) || !ok(cudaMalloc(&b->d_flag, sizeof(unsigned int) * n)) ||
      !ok(cudaMalloc(&b->d_bar, sizeof(unsigned int) * 4)) || !ok(cudaMalloc(&b->stage, sizeof(double) * 18 * big)))
    return fail("tables");
  if (!ok(cudaMemcpy(b->d_off, b->off.data(), sizeof(long long) * n, cudaMemcpyHostToDevice)) ||
      !ok(cudaMemcpy(b->d_nx, b->nx.data(), sizeof(int) * n, cudaMemcpyHostToDevice)) ||
      !ok(cudaMemcpy(b->d_ny, b->ny.data(), sizeof(int) * n, cudaMemcpyHostToDevice)) ||
      !ok(cudaMemcpy(b->d_dtau, b->dtau.data(), sizeof(double) * n, cudaMemcpyHostToDevice)) ||
      !ok(cudaMemcpy(b->d_taumax, b->tau_max.data(), sizeof(double) * n, cudaMemcpyHostToDevice)))
    return fail("tables");
  b->t_freeze_gev = t_freeze_gev;
  if (vh_batch_reset(b) != VH_OK) return fail("reset");
  if (build_items(b) != VH_OK) return fail("items");
  *out = b;
  return VH_OK;
}

extern "C" int vh_batch_reset(vh_batch* b) {
  if (!b) return VH_E_ARG;
  const int n = b->n;
  std::vector<int> zeros(n, 0);
  VB_CUDA(b, cudaMemcpy(b->d_tau, b->tau0.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
  VB_CUDA(b, cudaMemcpy(b->d_state, zeros.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  VB_CUDA(b, cudaMemcpy(b->d_steps, zeros.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  VB_CUDA(b, cudaMemset(b->d_tmax, 0, sizeof(unsigned long long) * n));
  VB_CUDA(b, cudaMemset(b->d_flag, 0, sizeof(unsigned int) * n));
  VB_CUDA(b, cudaMemset(b->d_bar, 0, sizeof(unsigned int) * 4));
  VB_CUDA(b, cudaMemset(b->d_iters, 0, sizeof(unsigned long long)));
  VB_CUDA(b, cudaMemcpy(b->d_running, &n, sizeof(int), cudaMemcpyHostToDevice));
  return VH_OK;
}

extern "C" int vh_batch_destroy(vh_batch* b) {
  if (!b) return VH_OK;
  cudaFree(b->pool); cudaFree(b->eos_d); cudaFree(b->eos_f);
  cudaFree(b->d_off); cudaFree(b->d_nx); cudaFree(b->d_ny); cudaFree(b->d_state); cudaFree(b->d_steps);
  cudaFree(b->d_running); cudaFree(b->d_tau); cudaFree(b->d_dtau); cudaFree(b->d_taumax); cudaFree(b->d_tmax);
  cudaFree(b->d_iters); cudaFree(b->d_flag); cudaFree(b->d_bar); cudaFree(b->stage);
  for (int q = 0; q < 2; q++) { cudaFree(b->d_x[q]); cudaFree(b->d_y[q]); }
  cudaFree(b->d_u);
  delete b;
  return VH_OK;
}

template <class R>
static int import_event(vh_batch* b, int ev, const double* host18, int pi_mode) {
  const long long n = (long long)(b->nx[ev] + 6) * (b->ny[ev] + 6);
  VB_CUDA(b, cudaMemcpy(b->stage, host18, sizeof(double) * 18 * n, cudaMemcpyHostToDevice));
  DevPtrs<R> P = pool_ptrs<R>(b).shifted(b->off[ev]);
  P.status = b->d_flag + ev;
  k_import_event<R><<<(unsigned)((n + 255) / 256), 256>>>(b->stage, P, n);
  DevCfg C = b->C0;
  C.nx = b->nx[ev]; C.ny = b->ny[ev]; C.gx = C.nx + 6; C.gy = C.ny + 6; C.px = C.gx; C.xt0 = 3; C.ir = 3 + C.nx; C.jr = 3 + C.ny;
  C.il = C.jl = 3; C.n = n;
  if (pi_mode == VH_PI_NS) {
    R* du16 = reinterpret_cast<R*>(b->stage);  // staging is free again after the import
    k_du_full<R><<<(unsigned)((n + 127) / 128), 128>>>(C, P, du16, b->dtau[ev]);
    k_ns_pi<R><<<(unsigned)((n + 127) / 128), 128>>>(C, P, du16, b->tau0[ev]);
  }
  k_fill_tmunu<R><<<(unsigned)((n + 255) / 256), 256>>>(C, P, b->tau0[ev]);
  VB_CUDA(b, cudaGetLastError());
  VB_CUDA(b, cudaDeviceSynchronize());
  return VH_OK;
}

extern "C" int vh_batch_init_event(vh_batch* b, int ev, const double* e, const double* ux, const double* uy,
                                   const double* prevu4, int pi_mode, const double* pi5) {
  if (!b || ev < 0 || ev >= b->n || !e || !ux || !uy) return VH_E_ARG;
  if (pi_mode != VH_PI_GIVEN && pi_mode != VH_PI_ZERO && pi_mode != VH_PI_NS) return VH_E_ARG;
  if (pi_mode == VH_PI_GIVEN && !pi5) return VH_E_ARG;
  const long long n = (long long)(b->nx[ev] + 6) * (b->ny[ev] + 6);
  std::vector<double> f(18 * (size_t)n, 0.0);
  for (long long c = 0; c < n; c++) {
    f[c] = e[c];
    f[2 * n + c] = ux[c];
    f[3 * n + c] = uy[c];
    f[n + c] = std::sqrt(1 + ux[c] * ux[c] + uy[c] * uy[c]);
    for (int l = 0; l < 5; l++) f[(5 + l) * n + c] = pi_mode == VH_PI_GIVEN ? pi5[l * n + c] : 0.0;
    for (int l = 0; l < 4; l++) f[(14 + l) * n + c] = prevu4 ? prevu4[l * n + c] : f[(1 + l) * n + c];
  }
  return b->mixed ? import_event<float>(b, ev, f.data(), pi_mode) : import_event<double>(b, ev, f.data(), pi_mode);
}

// Glauber events for every slot, generated on host threads (vh_profile_glauber
// per event with its seed and impact parameter), u = 0, pi = 0.
extern "C" int vh_batch_init_glauber(vh_batch* b, const uint64_t* seeds, const double* bimp, int A, double R,
                                     double aws, double dmin, double sigma_nn, double w, double epeak_gev,
                                     double efloor_gev, int nthreads, int* npart_out) {
  if (!b || !seeds || !bimp) return VH_E_ARG;
  const int n = b->n;
  std::vector<std::vector<double>> es(n);
  std::vector<int> np(n, 0);
  int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
  nt = std::min(nt, n);
  std::vector<std::thread> th;
  std::vector<int> rc(nt, VH_OK);
  for (int t = 0; t < nt; t++)
    th.emplace_back([&, t]() {
      for (int ev = t; ev < n; ev += nt) {
        es[ev].assign((size_t)(b->nx[ev] + 6) * (b->ny[ev] + 6), 0.0);
        int r = vh_profile_glauber(b->nx[ev], b->ny[ev], 1, 1, b->cfg.dx, b->cfg.dy, 1.0, A, R, aws, dmin, bimp[ev],
                                   sigma_nn, w, epeak_gev, 0.0, 1.0, efloor_gev, b->cfg.hbarc, seeds[ev],
                                   es[ev].data(), &np[ev]);
        if (r) rc[t] = r;
      }
    });
  for (auto& x : th) x.join();
  for (int r : rc) if (r) return r;
  for (int ev = 0; ev < n; ev++) {
    std::vector<double> z(es[ev].size(), 0.0);
    if (int r = vh_batch_init_event(b, ev, es[ev].data(), z.data(), z.data(), nullptr, VH_PI_ZERO, nullptr)) return r;
    if (npart_out) npart_out[ev] = np[ev];
  }
  return VH_OK;
}

template <class R, int NC, int MINB, int UNR>
static int launch_variant(vh_batch* b, cudaStream_t s, int nsteps, bool query_only, int* max_blocks) {
  using SX = DirSmem<R, 0, NC>;
  using SY = DirSmem<R, 1, NC>;
  const size_t sm = std::max(sizeof(SX), sizeof(SY));
  auto kern = k_batch<R, NC, MINB, UNR>;
  VB_CUDA(b, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  int per_sm = 0, dev = 0, nsm = 0;
  VB_CUDA(b, cudaGetDevice(&dev));
  VB_CUDA(b, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  VB_CUDA(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NC * 32, sm));
  const int blocks = std::min(per_sm, MINB) * nsm;
  if (max_blocks) *max_blocks = blocks;
  if (query_only) return blocks > 0 ? VH_OK : VH_E_UNSUPPORTED;
  if (blocks <= 0) return VH_E_UNSUPPORTED;
  Args<R> A{};
  A.C0 = b->C0;
  A.pool = pool_ptrs<R>(b);
  Tables& T = A.T;
  T.n_events = b->n; T.off = b->d_off; T.nx = b->d_nx; T.ny = b->d_ny; T.tau = b->d_tau; T.dtau = b->d_dtau;
  T.tau_max = b->d_taumax; T.state = b->d_state; T.steps = b->d_steps; T.tmax_bits = b->d_tmax; T.flag = b->d_flag;
  const int q = NC == 4 ? 0 : 1;
  T.xitems = b->d_x[q]; T.n_x = b->n_xi[q]; T.yitems = b->d_y[q]; T.n_y = b->n_yi[q];
  T.uitems = b->d_u; T.n_u = b->n_ui; T.bar = b->d_bar; T.running = b->d_running; T.iters = b->d_iters;
  T.t_freeze_gev = b->t_freeze_gev;
  cudaLaunchConfig_t lc{};
  lc.gridDim = dim3(blocks);
  lc.blockDim = dim3(NC * 32);
  lc.dynamicSmemBytes = sm;
  lc.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  VB_CUDA(b, cudaLaunchKernelEx(&lc, kern, A, nsteps));
  return VH_OK;
}

static int launch(vh_batch* b, int variant, cudaStream_t s, int nsteps, bool query_only = false, int* blocks = nullptr) {
  if (b->mixed) {
    switch (variant) {
      case 0: return launch_variant<float, 4, 4, 1>(b, s, nsteps, query_only, blocks);
      case 1: return launch_variant<float, 4, 3, 1>(b, s, nsteps, query_only, blocks);
      case 2: return launch_variant<float, 8, 2, 1>(b, s, nsteps, query_only, blocks);
      case 3: return launch_variant<float, 8, 2, 3>(b, s, nsteps, query_only, blocks);
      default: return launch_variant<float, 8, 1, 1>(b, s, nsteps, query_only, blocks);
    }
  }
  switch (variant) {
    case 0: return launch_variant<double, 4, 4, 1>(b, s, nsteps, query_only, blocks);
    case 1: return launch_variant<double, 4, 3, 1>(b, s, nsteps, query_only, blocks);
    case 2: return launch_variant<double, 8, 2, 1>(b, s, nsteps, query_only, blocks);
    case 3: return launch_variant<double, 8, 2, 3>(b, s, nsteps, query_only, blocks);
    default: return launch_variant<double, 8, 1, 1>(b, s, nsteps, query_only, blocks);
  }
}

// Run until every event has stopped (or max_steps steps): launches of
// steps_per_launch steps each, recorded once into a CUDA graph of
// `per_graph` launches and replayed; the running count is read after each
// replay.  Returns the device seconds in *seconds.
extern "C" int vh_batch_run(vh_batch* b, int max_steps, double* seconds, int* graph_used) {
  if (!b || max_steps < 0) return VH_E_ARG;
  VhNvtxRange range("batched ensemble run");
  const int block = kVariants[b->variant].nc * 32;
  if (int r = build_uitems(b, block)) return r;
  cudaStream_t s;
  VB_CUDA(b, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  const int spl = b->steps_per_launch;
  const int per_graph = 4;
  cudaGraphExec_t exec = nullptr;
  bool graph = b->use_graph;
  if (graph) {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      int r = VH_OK;
      for (int q = 0; q < per_graph && !r; q++) r = launch(b, b->variant, s, spl);
      cudaError_t ec = cudaStreamEndCapture(s, &g);
      if (r || ec != cudaSuccess || cudaGraphInstantiate(&exec, g, 0) != cudaSuccess) { graph = false; exec = nullptr; }
      if (g) cudaGraphDestroy(g);
    } else {
      graph = false;
    }
    cudaGetLastError();  // clear a failed capture, if any
  }
  if (graph_used) *graph_used = graph ? 1 : 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s);
  int done_steps = 0, running = b->n, rc = VH_OK;
  while (done_steps < max_steps && running > 0) {
    if (graph && done_steps + spl * per_graph <= max_steps) {
      if (cudaGraphLaunch(exec, s) != cudaSuccess) { rc = VH_E_CUDA; break; }
      done_steps += spl * per_graph;
    } else {
      const int k = std::min(spl, max_steps - done_steps);
      if ((rc = launch(b, b->variant, s, k))) break;
      done_steps += k;
    }
    // the running count and the sticky barrier time-out flag together: after
    // a time-out every later launch returns at its first barrier, so the
    // loop stops at once instead of launching until max_steps
    unsigned int flag = 0;
    if (cudaMemcpyAsync(&running, b->d_running, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(&flag, b->d_bar + 2, sizeof(flag), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) { rc = VH_E_CUDA; b->err = cudaGetErrorString(cudaGetLastError()); break; }
    if (flag) break;
  }
  cudaEventRecord(e1, s);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  if (seconds) *seconds = ms / 1e3;
  unsigned int bar[4] = {0, 0, 0, 0};
  cudaMemcpy(bar, b->d_bar, sizeof(bar), cudaMemcpyDeviceToHost);
  if (exec) cudaGraphExecDestroy(exec);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(s);
  if (rc) return rc;
  if (bar[2]) { b->err = "grid barrier timed out"; return VH_E_TIMEOUT; }
  return VH_OK;
}

extern "C" int vh_batch_events(vh_batch* b, double* tau, int* steps, int* state) {
  if (!b) return VH_E_ARG;
  const int n = b->n;
  if (tau) VB_CUDA(b, cudaMemcpy(tau, b->d_tau, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (steps) VB_CUDA(b, cudaMemcpy(steps, b->d_steps, sizeof(int) * n, cudaMemcpyDeviceToHost));
  if (state) VB_CUDA(b, cudaMemcpy(state, b->d_state, sizeof(int) * n, cudaMemcpyDeviceToHost));
  return VH_OK;
}

extern "C" int vh_batch_get_event_state(vh_batch* b, int ev, double* host18) {
  if (!b || ev < 0 || ev >= b->n || !host18) return VH_E_ARG;
  const long long n = (long long)(b->nx[ev] + 6) * (b->ny[ev] + 6);
  if (b->mixed) {
    DevPtrs<float> P = pool_ptrs<float>(b).shifted(b->off[ev]);
    k_export_event<float><<<(unsigned)((n + 255) / 256), 256>>>(P, b->stage, n);
  } else {
    DevPtrs<double> P = pool_ptrs<double>(b).shifted(b->off[ev]);
    k_export_event<double><<<(unsigned)((n + 255) / 256), 256>>>(P, b->stage, n);
  }
  VB_CUDA(b, cudaGetLastError());
  VB_CUDA(b, cudaMemcpy(host18, b->stage, sizeof(double) * 18 * n, cudaMemcpyDeviceToHost));
  return VH_OK;
}

extern "C" int vh_batch_set_tuning(vh_batch* b, int variant, int steps_per_launch, int use_graph) {
  if (!b || variant < 0 || variant >= kNumVariants || steps_per_launch < 1) return VH_E_ARG;
  b->variant = variant;
  b->steps_per_launch = steps_per_launch;
  b->use_graph = use_graph != 0;
  return VH_OK;
}

extern "C" int vh_batch_get_tuning(vh_batch* b, int* variant, int* steps_per_launch, int* nc, int* minb, int* unroll) {
  if (!b) return VH_E_ARG;
  if (variant) *variant = b->variant;
  if (steps_per_launch) *steps_per_launch = b->steps_per_launch;
  if (nc) *nc = kVariants[b->variant].nc;
  if (minb) *minb = kVariants[b->variant].minb;
  if (unroll) *unroll = kVariants[b->variant].unr;
  return VH_OK;
}

// Autotuner: time `probe_steps` steps of every compiled variant x
// steps-per-launch choice from the current state (the pool and tables are
// saved before and restored after each trial), keep the fastest, and cache
// the choice in cache_path under a key of device, precision and event-size
// histogram (an existing entry is reused without timing).
extern "C" int vh_batch_autotune(vh_batch* b, const char* cache_path, int probe_steps, double* best_ms_per_step) {
  if (!b || probe_steps < 1) return VH_E_ARG;
  int dev = 0;
  cudaDeviceProp prop{};
  VB_CUDA(b, cudaGetDevice(&dev));
  VB_CUDA(b, cudaGetDeviceProperties(&prop, dev));
  long long hist[5] = {0, 0, 0, 0, 0};
  for (int e = 0; e < b->n; e++) hist[std::min(4, (b->nx[e] * b->ny[e]) / 10000)]++;
  std::ostringstream key;
  key << prop.name << "|" << (b->mixed ? "mixed" : "fp64") << "|" << b->n;
  for (long long h : hist) key << ":" << h;
  if (cache_path) {
    std::ifstream in(cache_path);
    std::string line;
    while (std::getline(in, line)) {
      const size_t sep = line.rfind('=');
      if (sep != std::string::npos && line.substr(0, sep) == key.str()) {
        int v = 0, spl = 0;
        if (sscanf(line.c_str() + sep + 1, "%d,%d", &v, &spl) == 2 && v >= 0 && v < kNumVariants && spl > 0) {
          b->variant = v;
          b->steps_per_launch = spl;
          if (best_ms_per_step) *best_ms_per_step = -1;
          return VH_OK;
        }
      }
    }
  }
  // save the state the trials will advance
  const size_t pool_bytes = (size_t)52 * b->ntot * b->esz;
  void* save = nullptr;
  VB_CUDA(b, cudaMalloc(&save, pool_bytes));
  // put the saved pool back; on failure free the copy and report
  auto restore = [&]() {
    const cudaError_t e = cudaMemcpy(b->pool, save, pool_bytes, cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) {
      b->err = std::string("vh_batch_autotune: restoring the pool: ") + cudaGetErrorString(e);
      cudaFree(save);
    }
    return e == cudaSuccess;
  };
  if (const cudaError_t e = cudaMemcpy(save, b->pool, pool_bytes, cudaMemcpyDeviceToDevice); e != cudaSuccess) {
    b->err = std::string("vh_batch_autotune: saving the pool: ") + cudaGetErrorString(e);
    cudaFree(save);
    return VH_E_CUDA;
  }
  double best = 1e300;
  int best_v = b->variant, best_s = b->steps_per_launch;
  for (int v = 0; v < kNumVariants; v++)
    for (int spl : kStepsChoices) {
      int blocks = 0;
      if (launch(b, v, 0, 0, true, &blocks) != VH_OK || blocks <= 0) continue;
      if (!restore()) return VH_E_CUDA;
      if (vh_batch_reset(b) != VH_OK) break;
      b->variant = v;
      b->steps_per_launch = spl;
      b->use_graph = false;
      const int steps = ((probe_steps + spl - 1) / spl) * spl;
      double sec = 0;
      if (vh_batch_run(b, spl, nullptr, nullptr) != VH_OK) continue;  // warm-up launch
      if (!restore()) return VH_E_CUDA;
      if (vh_batch_reset(b) != VH_OK) break;
      if (vh_batch_run(b, steps, &sec, nullptr) != VH_OK) continue;
      const double ms = 1e3 * sec / steps;
      if (ms < best) { best = ms; best_v = v; best_s = spl; }
    }
  if (!restore()) return VH_E_CUDA;
  cudaFree(save);
  vh_batch_reset(b);
  b->variant = best_v;
  b->steps_per_launch = best_s;
  b->use_graph = true;
  if (best_ms_per_step) *best_ms_per_step = best;
  if (cache_path && best < 1e300) {
    std::ofstream out(cache_path, std::ios::app);
    out << key.str() << "=" << best_v << "," << best_s << "\n";
  }
  return VH_OK;
}

extern "C" int vh_batch_barrier_selftest(int absent_blocks, double* seconds) {
  if (absent_blocks < 0 || absent_blocks > 1) return VH_E_ARG;
  unsigned int* bar = nullptr;
  if (cudaMalloc(&bar, 3 * sizeof(unsigned int)) != cudaSuccess) return VH_E_NOMEM;
  unsigned int h[3] = {0, 0, 0};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaError_t err = cudaMemset(bar, 0, 3 * sizeof(unsigned int));
  if (err == cudaSuccess) {
    cudaEventRecord(e0);
    k_barrier_probe<<<2, 32>>>(bar, absent_blocks);
    cudaEventRecord(e1);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) err = cudaMemcpy(h, bar, sizeof(h), cudaMemcpyDeviceToHost);
  float ms = 0;
  if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(bar);
  if (err != cudaSuccess) {
    g_batch_err = std::string("vh_batch_barrier_selftest: ") + cudaGetErrorString(err);
    return VH_E_CUDA;
  }
  if (seconds) *seconds = ms / 1e3;
  if (h[2]) {
    g_batch_err = "grid barrier timed out";
    return VH_E_TIMEOUT;
  }
  return VH_OK;
}

// Per-event observables of the current states, one block per event, FP64
// sums in a fixed order: the momentum anisotropy
// eps_p = sum(T^xx - T^yy) / sum(T^xx + T^yy) and the eccentricity of the
// energy density about its centre,
// eps_2 = sqrt((<y^2> - <x^2>)^2 + 4 <xy>^2) / (<x^2> + <y^2>).
template <class R>
__global__ void __launch_bounds__(256) k_batch_obs(DevCfg C0, DevPtrs<R> pool, const long long* off, const int* nx,
                                                   const int* ny, double* out) {
  const int ev = blockIdx.x;
  const DevCfg C = event_cfg(C0, nx[ev], ny[ev]);
  const DevPtrs<R> P = pool.shifted(off[ev]);
  const long long nint = (long long)C.nx * C.ny;
  double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // N, D, sum e, e x, e y, e x^2, e y^2, e x y
  for (long long t = threadIdx.x; t < nint; t += blockDim.x) {
    const int i = (int)(t % C.nx), j = (int)(t / C.nx);
    const long long c = cix(C, C.il + i, C.jl + j, 0);
    const R e = P.e()[c];
    double num, den;
    obs_cell<R>(C, e, P.u(1)[c], P.u(2)[c], P.A(4)[c], P.A(5)[c], num, den);
    const double x = i * C.dx, y = j * C.dy, ed = (double)e;
    s[0] += num; s[1] += den; s[2] += ed; s[3] += ed * x; s[4] += ed * y;
    s[5] += ed * x * x; s[6] += ed * y * y; s[7] += ed * x * y;
  }
  __shared__ double sh[8][256];
#pragma unroll
  for (int q = 0; q < 8; q++) sh[q][threadIdx.x] = s[q];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
#pragma unroll
      for (int q = 0; q < 8; q++) sh[q][threadIdx.x] += sh[q][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double E = sh[2][0], xm = sh[3][0] / E, ym = sh[4][0] / E;
    const double xx = sh[5][0] / E - xm * xm, yy = sh[6][0] / E - ym * ym, xy = sh[7][0] / E - xm * ym;
    out[2 * ev] = sh[0][0] / sh[1][0];
    out[2 * ev + 1] = sqrt((yy - xx) * (yy - xx) + 4 * xy * xy) / (xx + yy);
  }
}

extern "C" int vh_batch_observables(vh_batch* b, double* eps_p, double* ecc2) {
  if (!b) return VH_E_ARG;
  double* d = nullptr;
  VB_CUDA(b, cudaMalloc(&d, sizeof(double) * 2 * b->n));
  if (b->mixed)
    k_batch_obs<float><<<b->n, 256>>>(b->C0, pool_ptrs<float>(b), b->d_off, b->d_nx, b->d_ny, d);
  else
    k_batch_obs<double><<<b->n, 256>>>(b->C0, pool_ptrs<double>(b), b->d_off, b->d_nx, b->d_ny, d);
  cudaError_t e = cudaGetLastError();
  std::vector<double> h(2 * (size_t)b->n);
  if (e == cudaSuccess) e = cudaMemcpy(h.data(), d, sizeof(double) * h.size(), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    b->err = std::string("vh_batch_observables: ") + cudaGetErrorString(e);
    return VH_E_CUDA;
  }
  for (int ev = 0; ev < b->n; ev++) {
    if (eps_p) eps_p[ev] = h[2 * ev];
    if (ecc2) ecc2[ev] = h[2 * ev + 1];
  }
  return VH_OK;
}

extern "C" const char* vh_batch_last_error(const vh_batch* b) { return b ? b->err.c_str() : g_batch_err.c_str(); }
