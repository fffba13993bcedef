// vh_step_static: the FP64 time step on caller-owned device memory, with all
// of the step's scratch in one file-scope device array, so that the call
// allocates nothing.
//
// Who needs it: callers that must not call cudaMalloc on the device at the
// point where they step the fluid.  The typical case is a host code whose
// device memory is owned by another framework's pool allocator: a cudaMalloc
// behind the pool's back fragments the device or exceeds the budget the pool
// was given.  Such a caller keeps the 18-field state in memory it owns and
// lends it to this call; the scratch the step needs (the stage-1 conserved
// set, the RK2 buffer, the flux-divergence and velocity-gradient
// accumulators and two status words) lives in g_vh_static_scratch below.
//
// Limits and sharing rules:
//  - FP64 only, at most VH_STATIC_MAX_CELLS ghost-inclusive cells
//    (34 scratch arrays x 61,680 doubles = 16 MiB); larger grids are
//    rejected with VH_E_ARG before anything runs.
//  - Every GPU that loads libvh holds the array until the process exits.
//  - All calls share the array and it keeps the last call's contents; the
//    status words are cleared at the start of every call.  Calls that
//    overlap on the GPU (two streams, two host threads) race on it: issue
//    them one after another.
//  - The first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and sets the kernels'
//    shared-memory attributes.
//  - Each call ends by copying the status word to the host and
//    synchronising the stream it was given, so it returns only once its
//    steps have finished on the GPU.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "vh.h"
#include "vh_kernels.cuh"

using namespace vh;

namespace {

constexpr long long kStaticArrays = 34;  // B(9) + v1t(4) + res(9) + du(12)
constexpr long long kStaticCells = VH_STATIC_MAX_CELLS;
constexpr long long kHeaderDoubles = 32;  // status word and iteration counter

static __device__ __align__(256) double g_vh_static_scratch[kHeaderDoubles + kStaticArrays * kStaticCells];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// once per device, with that device current
int static_setup(int dev, double** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_vh_static_scratch) != cudaSuccess || !p) return VH_E_CUDA;
    if (cudaFuncSetAttribute(k_dir<double, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(DirSmem<double, 0>)) != cudaSuccess ||
        cudaFuncSetAttribute(k_dir<double, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(DirSmem<double, 1>)) != cudaSuccess ||
        cudaFuncSetAttribute(k_dir<double, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(DirSmem<double, 2>)) != cudaSuccess)
      return VH_E_CUDA;
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return VH_OK;
}

int fill_cfg(const vh_config* c, const double* eos_dev, double tau, DevCfg& C) {
  if (!c || c->precision != VH_PREC_FP64) return VH_E_ARG;
  // Milne sources divide by tau (the time is a call argument here, not
  // cfg->tau0)
  if (!std::isfinite(tau) || (c->coords == VH_COORD_MILNE && !(tau > 0))) return VH_E_ARG;
  if (c->coords != VH_COORD_MILNE && c->coords != VH_COORD_CARTESIAN) return VH_E_ARG;
  if (c->recon != VH_RECON_WENO5 && c->recon != VH_RECON_MINMOD) return VH_E_ARG;
  if (c->nx < 3 || c->ny < 3 || (!c->boost_invariant && c->nz < 3) || (c->boost_invariant && c->nz != 1)) return VH_E_ARG;
  if (!(c->dx > 0 && c->dy > 0 && (c->boost_invariant || c->dz > 0) && c->dtau > 0)) return VH_E_ARG;
  if (c->taupi_kind != VH_TAUPI_15_ETA_OVER_P && c->taupi_kind != VH_TAUPI_5_ETA_OVER_EPP) return VH_E_ARG;
  if (c->cold_plasma) return VH_E_ARG;  // the test mode runs through vh_step only
  C = DevCfg{};
  C.nx = c->nx; C.ny = c->ny; C.nz = c->boost_invariant ? 1 : c->nz;
  C.gx = c->nx + 2 * NG; C.gy = c->ny + 2 * NG; C.gz = c->boost_invariant ? 1 : c->nz + 2 * NG;
  C.px = C.gx;  // the caller's state is in the canonical, unpadded layout
  C.xt0 = NG;
  C.il = NG; C.ir = NG + c->nx; C.jl = NG; C.jr = NG + c->ny;
  C.kl = c->boost_invariant ? 0 : NG; C.kr = c->boost_invariant ? 1 : NG + c->nz;
  C.n = (long long)C.gx * C.gy * C.gz;
  C.cart = c->coords == VH_COORD_CARTESIAN;
  C.bi = c->boost_invariant != 0;
  C.recon = c->recon;
  C.mirror = c->gubser_mirror != 0;
  C.dx = c->dx; C.dy = c->dy; C.dz = c->boost_invariant ? 1.0 : c->dz;
  C.eos_kind = c->eos_kind; C.eos_a = c->eos_a;
  C.etas0 = c->etas0; C.etas1 = c->etas1; C.etas_tc = c->etas_tc; C.hbarc = c->hbarc;
  C.taupi_kind = c->taupi_kind;
  C.mm_theta = c->minmod_theta;
  if (c->eos_kind == VH_EOS_CONFORMAL) {
    if (!(c->eos_a > 0)) return VH_E_ARG;
  } else if (c->eos_kind == VH_EOS_TABLE) {
    if (c->eos_n < 2 || !c->eos_e || !eos_dev) return VH_E_ARG;
    // the table lookup brackets e by its logarithm: the rows must increase
    for (int i = 1; i < c->eos_n; i++)
      if (!(c->eos_e[i] > c->eos_e[i - 1]) || !(c->eos_e[i - 1] > 0)) return VH_E_ARG;
    C.eos_n = c->eos_n;
    C.eos_l0 = std::log(c->eos_e[0]);
    C.eos_idl = (c->eos_n - 1) / (std::log(c->eos_e[c->eos_n - 1]) - C.eos_l0);
    C.eos_d = eos_dev;
  } else {
    return VH_E_ARG;
  }
  return VH_OK;
}

int launch_dir_static(const DevCfg& C, const DevPtrs<double>& P, int dir, int use_b, double tau, int first,
                      cudaStream_t s) {
  const int nzi = C.kr - C.kl;
  const double hh = dir == 0 ? C.dx : (dir == 1 ? C.dy : C.dz);
  if (dir == 0) {
    using T = Tile<0, double>;
    dim3 grid((C.nx + T::NA - 7) / (T::NA - 6), (C.ny + T::NC - 1) / T::NC, nzi);
    k_dir<double, 0><<<grid, dim3(T::NA * T::NC), sizeof(DirSmem<double, 0>), s>>>(C, P, use_b, tau, 1.0 / hh, hh, first);
  } else if (dir == 1) {
    using T = Tile<1, double>;
    dim3 grid((C.ny + T::NA - 7) / (T::NA - 6), (C.ir - C.xt0 + T::NC - 1) / T::NC, nzi);
    k_dir<double, 1><<<grid, dim3(T::NA * T::NC), sizeof(DirSmem<double, 1>), s>>>(C, P, use_b, tau, 1.0 / hh, hh, first);
  } else {
    using T = Tile<2, double>;
    dim3 grid((C.nz + T::NA - 7) / (T::NA - 6), (C.ir - C.xt0 + T::NC - 1) / T::NC, C.ny);
    k_dir<double, 2><<<grid, dim3(T::NA * T::NC), sizeof(DirSmem<double, 2>), s>>>(C, P, use_b, tau, 1.0 / hh, hh, first);
  }
  return cudaGetLastError() == cudaSuccess ? VH_OK : VH_E_CUDA;
}

}  // namespace

extern "C" int vh_step_static(const vh_config* cfg, double* state, const double* eos_dev, double tau, int nsteps,
                              void* stream) {
  DevCfg C;
  if (!state || nsteps < 0) return VH_E_ARG;
  if (fill_cfg(cfg, eos_dev, tau, C) != VH_OK) return VH_E_ARG;
  if (C.n > kStaticCells) return VH_E_ARG;  // grid larger than the static scratch
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return VH_E_CUDA;
  double* scratch = nullptr;
  if (int r = static_setup(dev, &scratch)) return r;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  DevPtrs<double> P{};
  const long long n = C.n;
  P.base0 = state;                           // the caller's 18 fields
  P.base1 = scratch + kHeaderDoubles;        // B, v1t, res, du in the static array
  P.stride = n;
  P.status = reinterpret_cast<unsigned int*>(scratch);
  P.iters = reinterpret_cast<unsigned long long*>(scratch + 1);
  if (cudaMemsetAsync(scratch, 0, kHeaderDoubles * sizeof(double), s) != cudaSuccess) return VH_E_CUDA;

  const double ts = cfg->dtau;
  const long long nint = (long long)C.nx * C.ny * (C.kr - C.kl);
  const unsigned blocks = (unsigned)((nint + 127) / 128);
  for (int st = 0; st < nsteps; st++) {
    for (int stage = 0; stage < 2; stage++) {
      const double t = stage ? tau + ts : tau;
      for (int d = 0; d < (C.bi ? 2 : 3); d++)
        if (int r = launch_dir_static(C, P, d, stage, t, d == 0, s)) return r;
      if (stage == 0) k_update<double, 1><<<blocks, 128, 0, s>>>(C, P, tau, ts);
      else k_update<double, 2><<<blocks, 128, 0, s>>>(C, P, tau, ts);
      if (cudaGetLastError() != cudaSuccess) return VH_E_CUDA;
    }
    tau += ts;
  }
  unsigned int status = 0;
  if (cudaMemcpyAsync(&status, P.status, sizeof(status), cudaMemcpyDeviceToHost, s) != cudaSuccess) return VH_E_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return VH_E_CUDA;
  if (status & ST_ROOT) return VH_E_ROOTFIND;
  if (status & ST_NEGE) return VH_E_NEG_ENERGY;
  if (status & ST_CAUSAL) return VH_E_CAUSALITY;
  return VH_OK;
}
