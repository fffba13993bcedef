// Pieces shared by the discrete adjoints (boost-invariant and 3+1D): the
// workspace carve, the recording forward step, the phase clock, the
// observable's sums and the fixed-order sum of the per-cell parameter
// gradients.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "vh_adjoint.cuh"
#include "vh_handle.cuh"

namespace vh {

// Carves the adjoint's device buffers out of one allocation kept in the
// handle (grown when a call needs more), so repeated calls allocate nothing.
struct Carve {
  char* base = nullptr;
  size_t off = 0;
  template <class T>
  T* take(size_t count) {
    T* p = reinterpret_cast<T*>(base ? base + off : nullptr);
    off += (count * sizeof(T) + 255) / 256 * 256;
    return p;
  }
};

// One forward step that also records X_n (the state at the step start) and
// Y_n (e, u and the conserved set after stage 1); the launches are those of
// step_once.
template <class R>
static int record_step(vh_handle* h, const DevPtrs<R>& P, R* xrec, R* yrec) {
  const DevCfg& C = h->C;
  const size_t nb = (size_t)C.n * sizeof(R);
  const double tau = h->tau, ts = h->cfg.dtau;
  cudaStream_t st = h->stream;
  int r;
  VH_CUDA(h, cudaMemcpyAsync(xrec, P.base0, 18 * nb, cudaMemcpyDeviceToDevice, st));
  if ((r = stage_rhs<R>(h, P, 0, tau))) return r;
  if ((r = stage_update<R, 1>(h, P, tau, ts))) return r;
  VH_CUDA(h, cudaMemcpyAsync(yrec, P.base0, 5 * nb, cudaMemcpyDeviceToDevice, st));
  VH_CUDA(h, cudaMemcpyAsync(yrec + 5 * C.n, P.base1, 9 * nb, cudaMemcpyDeviceToDevice, st));
  if ((r = stage_rhs<R>(h, P, 1, tau + ts))) return r;
  if ((r = stage_update<R, 2>(h, P, tau, ts))) return r;
  h->tau = tau + ts;
  return VH_OK;
}

// events bracketing the phases of one call, read once at its end
struct PhaseClock {
  std::vector<cudaEvent_t> ev;
  ~PhaseClock() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
  }
  cudaError_t mark(cudaStream_t s, int* idx) {
    cudaEvent_t e;
    cudaError_t r = cudaEventCreate(&e);
    if (r != cudaSuccess) return r;
    ev.push_back(e);
    *idx = (int)ev.size() - 1;
    return cudaEventRecord(e, s);
  }
  float ms(int a, int b) const {
    float t = 0;
    cudaEventElapsedTime(&t, ev[a], ev[b]);
    return t;
  }
};

// momentum anisotropy: per-block partial sums of T^xx - T^yy and T^xx + T^yy
// over the interior cells (every eta slice of a 3+1D grid), then one
// fixed-order sum (deterministic)
constexpr int kObsBlocks = 148;
template <class R>
__global__ void __launch_bounds__(256) k_obs_part(DevCfg C, const R* S, long long n, double* part) {
  double a = 0, b = 0;
  const long long nint = (long long)C.nx * C.ny * C.nz;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nint;
       t += (long long)gridDim.x * blockDim.x) {
    const long long c = cell_at(C, t).c;
    double num, den;
    obs_cell<R>(C, S[c], S[2 * n + c], S[3 * n + c], S[5 * n + c], S[6 * n + c], num, den);
    a += num;
    b += den;
  }
  __shared__ double sa[8], sb[8];
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) { sa[threadIdx.x >> 5] = a; sb[threadIdx.x >> 5] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0, tb = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) { ta += sa[w]; tb += sb[w]; }
    part[2 * blockIdx.x] = ta;
    part[2 * blockIdx.x + 1] = tb;
  }
}
static __global__ void k_obs_final(const double* part, int nb, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double a = 0, b = 0;
    for (int k = 0; k < nb; k++) { a += part[2 * k]; b += part[2 * k + 1]; }
    out[0] = a;
    out[1] = b;
  }
}


// the two per-cell parameter-gradient arrays summed in a fixed order (so the
// gradient is reproducible): kObsBlocks contiguous chunks, each reduced by a
// tree in its block, then the chunk sums in order
static __global__ void __launch_bounds__(256) k_sum_part(const double* cacc, long long n, double* part) {
  __shared__ double s0[256], s1[256];
  const long long chunk = (n + gridDim.x - 1) / gridDim.x;
  const long long c0 = (long long)blockIdx.x * chunk, c1 = c0 + chunk < n ? c0 + chunk : n;
  double a = 0, b = 0;
  for (long long c = c0 + threadIdx.x; c < c1; c += blockDim.x) { a += cacc[c]; b += cacc[n + c]; }
  s0[threadIdx.x] = a;
  s1[threadIdx.x] = b;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) { s0[threadIdx.x] += s0[threadIdx.x + w]; s1[threadIdx.x] += s1[threadIdx.x + w]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = s0[0]; part[2 * blockIdx.x + 1] = s1[0]; }
}
// cacc: 2 x n per-cell sums; part: 2 x kObsBlocks scratch; out2: the totals
static inline void sum_cells(const double* cacc, long long n, double* part, double* out2, cudaStream_t st) {
  k_sum_part<<<kObsBlocks, 256, 0, st>>>(cacc, n, part);
  k_obs_final<<<1, 32, 0, st>>>(part, kObsBlocks, out2);
}

template <class R>
static int eps_p_device(vh_handle* h, const R* S, double* part, double* nd_dev, double* nd_host) {
  const DevCfg& C = h->C;
  k_obs_part<R><<<kObsBlocks, 256, 0, h->stream>>>(C, S, C.n, part);
  k_obs_final<<<1, 32, 0, h->stream>>>(part, kObsBlocks, nd_dev);
  VH_CUDA(h, cudaGetLastError());
  if (nd_host) {
    VH_CUDA(h, cudaMemcpyAsync(nd_host, nd_dev, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    VH_CUDA(h, cudaStreamSynchronize(h->stream));
  }
  return VH_OK;
}


// the 3+1D discrete adjoint (vh_adjoint3.cu)
int adjoint3_eps_p(vh_handle* h, int nsteps, int every, double* eps_p, double* grad_state, double* grad_e,
                   double* grad_etas);

}  // namespace vh
