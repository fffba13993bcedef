// The handle behind the C ABI and the launch sequence of one TVDRK2 step,
// shared by the translation units that drive the step (the entry points of
// include/vh.h and the discrete adjoint).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "vh.h"
#include "vh_aux.cuh"
#include "vh_nvtx.h"

using namespace vh;

struct vh_handle {
  vh_config cfg{};
  DevCfg C{};
  cudaStream_t stream = nullptr;
  bool mixed = false;
  size_t esz = 8;            // bytes per state element
  void* state = nullptr;     // 18 canonical fields + B(9) + v1t(4) + res(9) + du(12)
  double* stage = nullptr;   // 18*n doubles: host<->device staging for the mixed path / du16 scratch
  double* eos_d = nullptr;
  float* eos_f = nullptr;
  unsigned int* status = nullptr;
  unsigned long long* iters = nullptr;
  unsigned long long* red = nullptr;  // reduction slots
  double* part = nullptr;              // conservation partial sums
  int part_blocks = 0;
  DevPtrs<double> pd{};
  DevPtrs<float> pf{};
  std::vector<double> eos_host;  // 4 x eos_n
  double tau = 0;
  bool have_state = false;
  // step kernels launched with programmatic dependent launch (VH_PDL=0 in
  // the environment at vh_create turns it off, e.g. under a profiler that
  // replays kernels one by one)
  bool pdl = true;
  // discrete-adjoint workspace (kept between calls) and the device
  // milliseconds of the last call's phases
  void* adj_buf = nullptr;
  size_t adj_bytes = 0;
  double adj_ms[4] = {0, 0, 0, 0};
  // the slice vh_freezeout_step saw last: T and u^mu (5 x n doubles) at
  // fo_tau; forgotten whenever the state is set from outside
  double* fo_prev = nullptr;
  double fo_tau = 0;
  bool fo_have = false;
  std::string err;
};

#define VH_CUDA(h, call)                                                                        \
  do {                                                                                          \
    cudaError_t _e = (call);                                                                    \
    if (_e != cudaSuccess) {                                                                    \
      (h)->err = std::string(#call) + ": " + cudaGetErrorString(_e);                            \
      return VH_E_CUDA;                                                                         \
    }                                                                                           \
  } while (0)

static inline int fail(vh_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

template <class R>
static void set_ptrs(DevPtrs<R>& P, void* base, long long n, unsigned int* status, unsigned long long* iters) {
  P.base0 = static_cast<R*>(base);
  P.base1 = static_cast<R*>(base) + 18 * n;
  P.stride = n;
  P.status = status;
  P.iters = iters;
}
static constexpr int kStateArrays = 52;

static inline unsigned grid1(long long n, int b) { return (unsigned)((n + b - 1) / b); }

// A step kernel launched with programmatic stream serialization (when pdl):
// it may begin while the kernel before it in the stream finishes its last
// blocks; the kernel itself waits for that kernel's completion before
// reading anything (pdl_wait_then_release), so the overlap covers launch and
// block set-up.
template <class K, class... Args>
static cudaError_t launch_step_kernel(bool pdl, K kernel, dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                      Args... args) {
  cudaLaunchConfig_t lc = {};
  lc.gridDim = grid;
  lc.blockDim = block;
  lc.dynamicSmemBytes = smem;
  lc.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&lc, kernel, args...);
}

template <class R>
static int launch_dir(vh_handle* h, const DevPtrs<R>& P, int dir, int use_b, double tau, int first) {
  const DevCfg& C = h->C;
  const int nzi = C.kr - C.kl;
  dim3 grid, block;
  size_t sm;
  const double hh = dir == 0 ? C.dx : (dir == 1 ? C.dy : C.dz);
  const R inv_h = (R)(1.0 / hh), hr = (R)hh;
  if (dir == 0) {
    using T = Tile<0, R>;
    block = dim3(T::NA * T::NC);
    grid = dim3((C.nx + T::NA - 7) / (T::NA - 6), (C.ny + T::NC - 1) / T::NC, nzi);
    sm = sizeof(DirSmem<R, 0>);
    VH_CUDA(h, launch_step_kernel(h->pdl, k_dir<R, 0>, grid, block, sm, h->stream, C, P, use_b, (R)tau, inv_h, hr,
                                  first));
  } else if (dir == 1) {
    using T = Tile<1, R>;
    block = dim3(T::NA * T::NC);
    grid = dim3((C.ny + T::NA - 7) / (T::NA - 6), (C.nx + T::NC - 1) / T::NC, nzi);
    sm = sizeof(DirSmem<R, 1>);
    VH_CUDA(h, launch_step_kernel(h->pdl, k_dir<R, 1>, grid, block, sm, h->stream, C, P, use_b, (R)tau, inv_h, hr,
                                  first));
  } else {
    using T = Tile<2, R>;
    block = dim3(T::NA * T::NC);
    grid = dim3((C.nz + T::NA - 7) / (T::NA - 6), (C.nx + T::NC - 1) / T::NC, C.ny);
    sm = sizeof(DirSmem<R, 2>);
    VH_CUDA(h, launch_step_kernel(h->pdl, k_dir<R, 2>, grid, block, sm, h->stream, C, P, use_b, (R)tau, inv_h, hr,
                                  first));
  }
  return VH_OK;
}

template <class R>
static int set_smem_attrs(vh_handle* h) {
  VH_CUDA(h, cudaFuncSetAttribute(k_dir<R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DirSmem<R, 0>)));
  VH_CUDA(h, cudaFuncSetAttribute(k_dir<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DirSmem<R, 1>)));
  VH_CUDA(h, cudaFuncSetAttribute(k_dir<R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DirSmem<R, 2>)));
  return VH_OK;
}

// the flux-divergence part of a stage: every direction into res, du
template <class R>
static int stage_rhs(vh_handle* h, const DevPtrs<R>& P, int use_b, double tau) {
  int r;
  if ((r = launch_dir<R>(h, P, 0, use_b, tau, 1))) return r;
  if ((r = launch_dir<R>(h, P, 1, use_b, tau, 0))) return r;
  if (!h->C.bi && (r = launch_dir<R>(h, P, 2, use_b, tau, 0))) return r;
  return VH_OK;
}

// the update part of a stage (sources, RK, root-find, ghosts): k_update,
// one thread per interior cell
template <class R, int STAGE>
static int stage_update(vh_handle* h, const DevPtrs<R>& P, double tau, double ts) {
  const DevCfg& C = h->C;
  const long long nint = (long long)C.nx * C.ny * (C.kr - C.kl);
  VH_CUDA(h, launch_step_kernel(h->pdl, k_update<R, STAGE>, dim3(grid1(nint, 128)), dim3(128), 0, h->stream, C, P,
                                tau, ts));
  return VH_OK;
}

template <class R>
static int step_once(vh_handle* h, const DevPtrs<R>& P) {
  VhNvtxRange range("TVDRK2 step");
  const double tau = h->tau, ts = h->cfg.dtau;
  int r;
  if ((r = stage_rhs<R>(h, P, 0, tau))) return r;
  if ((r = stage_update<R, 1>(h, P, tau, ts))) return r;
  if ((r = stage_rhs<R>(h, P, 1, tau + ts))) return r;
  if ((r = stage_update<R, 2>(h, P, tau, ts))) return r;
  h->tau = tau + ts;
  return VH_OK;
}


static inline int read_status(vh_handle* h) {
  unsigned int st = 0;
  VH_CUDA(h, cudaMemcpyAsync(&st, h->status, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  if (st & ST_ROOT) return fail(h, VH_E_ROOTFIND, "root-find failed in at least one cell");
  if (st & ST_NEGE) return fail(h, VH_E_NEG_ENERGY, "non-positive energy density after the root-find");
  if (st & ST_CAUSAL) return fail(h, VH_E_CAUSALITY, "superluminal velocity after the root-find");
  return VH_OK;
}
