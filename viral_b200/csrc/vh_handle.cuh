// The handle behind the C ABI and the launch sequence of one TVDRK2 step,
// shared by the translation units that drive the step (the entry points of
// include/vh.h and the discrete adjoint).
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
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
  // tensor maps of the state for the flux sweeps' TMA tiles, per direction:
  // [0] arrays 0..4 (e, u^mu), [1] a conserved set (9 arrays)
  alignas(64) CUtensorMap tmap[3][2];
  bool tma = false;         // the maps were made (else the sweeps load through the cache)
  bool tma_wanted = true;  // VH_TMA=0 in the environment at vh_create: cached loads
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
  // canonical-layout transfer buffer between host arrays and the padded
  // device arrays (allocated on first use)
  double* xfer = nullptr;
  size_t xfer_bytes = 0;
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
    if (h->tma)
      VH_CUDA(h, launch_step_kernel(h->pdl, k_dir_tma<R, 0>, grid, block, sm, h->stream, C, P, use_b, (R)tau, inv_h,
                                    hr, first, h->tmap[0][0], h->tmap[0][1]));
    else
      VH_CUDA(h, launch_step_kernel(h->pdl, k_dir<R, 0>, grid, block, sm, h->stream, C, P, use_b, (R)tau, inv_h, hr,
                                    first));
  } else if (dir == 1) {
    using T = Tile<1, R>;
    block = dim3(T::NA * T::NC);
    grid = dim3((C.ny + T::NA - 7) / (T::NA - 6), (C.ir - C.xt0 + T::NC - 1) / T::NC, nzi);
    sm = sizeof(DirSmem<R, 1>);
    if (h->tma)
      VH_CUDA(h, launch_step_kernel(h->pdl, k_dir_tma<R, 1>, grid, block, sm, h->stream, C, P, use_b, (R)tau, inv_h,
                                    hr, first, h->tmap[1][0], h->tmap[1][1]));
    else
      VH_CUDA(h, launch_step_kernel(h->pdl, k_dir<R, 1>, grid, block, sm, h->stream, C, P, use_b, (R)tau, inv_h, hr,
                                    first));
  } else {
    using T = Tile<2, R>;
    block = dim3(T::NA * T::NC);
    grid = dim3((C.nz + T::NA - 7) / (T::NA - 6), (C.ir - C.xt0 + T::NC - 1) / T::NC, C.ny);
    sm = sizeof(DirSmem<R, 2>);
    if (h->tma)
      VH_CUDA(h, launch_step_kernel(h->pdl, k_dir_tma<R, 2>, grid, block, sm, h->stream, C, P, use_b, (R)tau, inv_h,
                                    hr, first, h->tmap[2][0], h->tmap[2][1]));
    else
      VH_CUDA(h, launch_step_kernel(h->pdl, k_dir<R, 2>, grid, block, sm, h->stream, C, P, use_b, (R)tau, inv_h, hr,
                                    first));
  }
  return VH_OK;
}

// The tensor maps of the state: a 4D tensor (x over the padded row pitch,
// y, z, array) of the 52 arrays, one box shape per sweep direction and
// array count (TmaBox).  cuTensorMapEncodeTiled comes from the driver
// through the runtime's entry-point query.
template <class R, int DIR>
static int encode_dir_maps(vh_handle* h, PFN_cuTensorMapEncodeTiled_v12000 enc) {
  using B = TmaBox<R, DIR, Tile<DIR, R>::NC>;
  const DevCfg& C = h->C;
  const cuuint64_t dims[4] = {(cuuint64_t)C.px, (cuuint64_t)C.gy, (cuuint64_t)C.gz, (cuuint64_t)kStateArrays};
  const cuuint64_t strides[3] = {(cuuint64_t)C.px * sizeof(R), (cuuint64_t)C.px * C.gy * sizeof(R),
                                 (cuuint64_t)C.n * sizeof(R)};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  for (int q = 0; q < 2; q++) {
    const cuuint32_t box[4] = {(cuuint32_t)B::BX, (cuuint32_t)B::BY, (cuuint32_t)B::BZ, q ? 9u : 5u};
    const CUresult r = enc(&h->tmap[DIR][q], sizeof(R) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                           4, h->state, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return VH_E_CUDA;
  }
  return VH_OK;
}

// Sets h->tma when every map of the grid's directions was made; a grid the
// encoder refuses (none is known) steps with the sweeps loading through the
// cache instead, the same arithmetic.
template <class R>
static void encode_maps(vh_handle* h) {
  h->tma = false;
  if (!h->tma_wanted) return;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn ||
      q != cudaDriverEntryPointSuccess) {
    cudaGetLastError();
    return;
  }
  auto enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  if (encode_dir_maps<R, 0>(h, enc) || encode_dir_maps<R, 1>(h, enc)) return;
  if (!h->C.bi && encode_dir_maps<R, 2>(h, enc)) return;
  h->tma = true;
}

template <class R>
static int set_smem_attrs(vh_handle* h) {
  VH_CUDA(h, cudaFuncSetAttribute(k_dir_tma<R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DirSmem<R, 0>)));
  VH_CUDA(h, cudaFuncSetAttribute(k_dir_tma<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DirSmem<R, 1>)));
  VH_CUDA(h, cudaFuncSetAttribute(k_dir_tma<R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DirSmem<R, 2>)));
  VH_CUDA(h, cudaFuncSetAttribute(k_dir<R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DirSmem<R, 0>)));
  VH_CUDA(h, cudaFuncSetAttribute(k_dir<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DirSmem<R, 1>)));
  VH_CUDA(h, cudaFuncSetAttribute(k_dir<R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DirSmem<R, 2>)));
  encode_maps<R>(h);
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


// Arrays of the C ABI (host or device memory) hold nfields fields of
// gx*gy*gz cells each, rows of gx cells; the handle's device arrays hold
// rows of px cells.  When the two differ, a kernel moves the rows between
// the layouts on the device: from (to) the caller's array itself when it is
// device memory, else through one contiguous copy to (from) the handle's
// transfer buffer, so that host data crosses the bus in a single copy.
static inline long long canon_cells(const DevCfg& C) { return (long long)C.gx * C.gy * C.gz; }

// TO_PAD: canonical src -> padded dst; else padded src -> canonical dst.
// One thread per canonical element.
template <bool TO_PAD>
static __global__ void k_repitch(const double* __restrict__ src, double* __restrict__ dst, long long total,
                                 long long nc, long long n, int gx, int px) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  const long long f = t / nc, r = t - f * nc, row = r / gx;
  const long long p = f * n + row * px + (r - row * gx);
  if (TO_PAD) dst[p] = src[t];
  else dst[t] = src[p];
}

static inline bool device_accessible(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// the transfer buffer, nfields canonical fields (allocated on first use)
static int xfer_buffer(vh_handle* h, int nfields, double** out) {
  const size_t need = sizeof(double) * (size_t)nfields * (size_t)canon_cells(h->C);
  if (h->xfer_bytes < need) {
    VH_CUDA(h, cudaStreamSynchronize(h->stream));
    cudaFree(h->xfer);
    h->xfer = nullptr;
    h->xfer_bytes = 0;
    VH_CUDA(h, cudaMalloc(&h->xfer, need));
    h->xfer_bytes = need;
  }
  *out = h->xfer;
  return VH_OK;
}

static int pitched_in(vh_handle* h, double* dev_padded, const double* canon, int nfields) {
  const DevCfg& C = h->C;
  const long long nc = canon_cells(C), total = nfields * nc;
  if (C.px == C.gx) {
    VH_CUDA(h, cudaMemcpyAsync(dev_padded, canon, sizeof(double) * total, cudaMemcpyDefault, h->stream));
    return VH_OK;
  }
  const double* src = canon;
  if (!device_accessible(canon)) {
    double* x = nullptr;
    if (int r = xfer_buffer(h, nfields, &x)) return r;
    VH_CUDA(h, cudaMemcpyAsync(x, canon, sizeof(double) * total, cudaMemcpyHostToDevice, h->stream));
    src = x;
  }
  k_repitch<true><<<grid1(total, 256), 256, 0, h->stream>>>(src, dev_padded, total, nc, C.n, C.gx, C.px);
  VH_CUDA(h, cudaGetLastError());
  return VH_OK;
}
static int pitched_out(vh_handle* h, double* canon, const double* dev_padded, int nfields) {
  const DevCfg& C = h->C;
  const long long nc = canon_cells(C), total = nfields * nc;
  if (C.px == C.gx) {
    VH_CUDA(h, cudaMemcpyAsync(canon, dev_padded, sizeof(double) * total, cudaMemcpyDefault, h->stream));
    return VH_OK;
  }
  if (device_accessible(canon)) {
    k_repitch<false><<<grid1(total, 256), 256, 0, h->stream>>>(dev_padded, canon, total, nc, C.n, C.gx, C.px);
    VH_CUDA(h, cudaGetLastError());
    return VH_OK;
  }
  double* x = nullptr;
  if (int r = xfer_buffer(h, nfields, &x)) return r;
  k_repitch<false><<<grid1(total, 256), 256, 0, h->stream>>>(dev_padded, x, total, nc, C.n, C.gx, C.px);
  VH_CUDA(h, cudaGetLastError());
  VH_CUDA(h, cudaMemcpyAsync(canon, x, sizeof(double) * total, cudaMemcpyDeviceToHost, h->stream));
  return VH_OK;
}

static inline int read_status(vh_handle* h) {
  unsigned int st = 0;
  VH_CUDA(h, cudaMemcpyAsync(&st, h->status, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
  VH_CUDA(h, cudaStreamSynchronize(h->stream));
  if (st & ST_ROOT) return fail(h, VH_E_ROOTFIND, "root-find failed in at least one cell");
  if (st & ST_NEGE) return fail(h, VH_E_NEG_ENERGY, "non-positive energy density after the root-find");
  if (st & ST_CAUSAL) return fail(h, VH_E_CAUSALITY, "superluminal velocity after the root-find");
  if (st & ST_TMA) return fail(h, VH_E_CUDA, "a flux-sweep tile copy (TMA) did not complete");
  return VH_OK;
}
