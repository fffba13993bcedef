// Isothermal freeze-out hypersurface and Cooper-Frye spectra on the GPU,
// from device arrays: the per-cube arithmetic of vh_freezeout.cuh, one
// thread per space-time cube, in two passes so that the elements land in the
// host entry points' order (cube order, x fastest) without atomics: a count
// pass from the signs of T - T_fo alone, an exclusive scan of the counts, and
// an emit pass in which each cut cube writes its elements from its offset.
// The spectra are a reduction over the elements per momentum bin, one block
// per bin with a fixed summation tree (deterministic).
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "vh.h"
#include "vh_freezeout.cuh"
#include "vh_nvtx.h"

namespace {

constexpr int kThreads = 256;

template <int D>
__global__ void __launch_bounds__(kThreads) k_fo_count(vh_fo::Geo g, const double* __restrict__ t0,
                                                        const double* __restrict__ t1, long long ncubes,
                                                        long long* __restrict__ counts) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncubes) return;
  int i, j, k;
  vh_fo::cube_ijk(g, c, &i, &j, &k);
  counts[c] = vh_fo::count<D>(g, i, j, k, t0, t1);
}

template <int D>
__global__ void __launch_bounds__(kThreads) k_fo_emit(vh_fo::Geo g, const double* __restrict__ t0,
                                                       const double* __restrict__ t1, const double* __restrict__ u0,
                                                       const double* __restrict__ u1, long long ncubes,
                                                       const long long* __restrict__ counts,
                                                       const long long* __restrict__ offs, double* __restrict__ out,
                                                       long long cap) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncubes || counts[c] == 0) return;
  int i, j, k;
  vh_fo::cube_ijk(g, c, &i, &j, &k);
  vh_fo::Sink s{out, offs[c], cap};  // writes below cap only
  if (D == 3)
    vh_fo::cube2(g, i, j, t0, t1, u0, u1, s);
  else
    vh_fo::cube3(g, i, j, k, t0, t1, u0, u1, s);
}

// one block per momentum bin (m_T, p_x, p_y); the block's threads stride
// over the elements and add their partial sums in a fixed tree
template <int D>
__global__ void __launch_bounds__(kThreads) k_cooper_frye(const double* __restrict__ el, long long count,
                                                           const double* __restrict__ bins, double y, double t_fo,
                                                           double pref, double* __restrict__ out) {
  __shared__ double red[kThreads];
  const long long b = blockIdx.x;
  const double mt = bins[3 * b], px = bins[3 * b + 1], py = bins[3 * b + 2];
  double s = 0;
  for (long long e = threadIdx.x; e < count; e += kThreads)
    s += D == 3 ? vh_fo::cf2_term(el + vh_fo::kW2 * e, mt, px, py, t_fo)
                : vh_fo::cf3_term(el + vh_fo::kW3 * e, mt, px, py, y, t_fo);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[b] = pref * red[0];
}

inline unsigned blocks(long long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// the surface between two device slices; scratch from the stream's pool
template <int D>
int surface(const vh_fo::Geo& g, const double* t0, const double* t1, const double* u0, const double* u1, double* out,
            long long cap, long long* count, cudaStream_t st) {
  const long long nc = vh_fo::cubes(g, D);
  if (nc > INT_MAX) return VH_E_ARG;  // one scan of int-counted items
  VhNvtxRange range("freeze-out surface");
  size_t scan_bytes = 0;
  const long long* scan_in = nullptr;
  long long* scan_out = nullptr;
  if (cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, scan_in, scan_out, (int)nc, st) != cudaSuccess)
    return VH_E_CUDA;
  const size_t words = 2 * (size_t)nc;  // counts, offsets
  char* buf = nullptr;
  if (cudaMallocAsync((void**)&buf, words * sizeof(long long) + scan_bytes + 256, st) != cudaSuccess) {
    cudaGetLastError();
    return VH_E_NOMEM;
  }
  long long* counts = reinterpret_cast<long long*>(buf);
  long long* offs = counts + nc;
  scan_in = counts;
  scan_out = offs;
  void* scan_tmp = buf + ((words * sizeof(long long) + 255) / 256) * 256;
  int rc = VH_OK;
  long long tail[2] = {0, 0};
  k_fo_count<D><<<blocks(nc), kThreads, 0, st>>>(g, t0, t1, nc, counts);
  if (cudaGetLastError() != cudaSuccess ||
      cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, scan_in, scan_out, (int)nc, st) != cudaSuccess ||
      cudaMemcpyAsync(&tail[0], offs + nc - 1, sizeof(long long), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(&tail[1], counts + nc - 1, sizeof(long long), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    rc = VH_E_CUDA;
  if (rc == VH_OK && cap > 0) {
    k_fo_emit<D><<<blocks(nc), kThreads, 0, st>>>(g, t0, t1, u0, u1, nc, counts, offs, out, cap);
    if (cudaGetLastError() != cudaSuccess) rc = VH_E_CUDA;
  }
  if (cudaFreeAsync(buf, st) != cudaSuccess && rc == VH_OK) rc = VH_E_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess && rc == VH_OK) rc = VH_E_CUDA;
  if (rc != VH_OK) return rc;
  *count = tail[0] + tail[1];
  return *count > cap ? VH_E_ARG : VH_OK;
}

// the spectrum of count device elements at the host's momentum bins
template <int D>
int spectrum(const double* el, long long count, double t_fo, double mass, double degeneracy, double y,
             const double* pt, int npt, const double* phi, int nphi, double* out, cudaStream_t st) {
  const long long nb = (long long)npt * nphi;
  if (nb > INT_MAX) return VH_E_ARG;
  VhNvtxRange range("Cooper-Frye spectrum");
  std::vector<double> bins(3 * (size_t)nb);
  for (int a = 0; a < npt; a++)
    for (int b = 0; b < nphi; b++) {
      double* q = &bins[3 * ((size_t)a * nphi + b)];
      q[0] = std::sqrt(mass * mass + pt[a] * pt[a]);
      q[1] = pt[a] * std::cos(phi[b]);
      q[2] = pt[a] * std::sin(phi[b]);
    }
  double* dbuf = nullptr;
  if (cudaMallocAsync((void**)&dbuf, 4 * (size_t)nb * sizeof(double), st) != cudaSuccess) {
    cudaGetLastError();
    return VH_E_NOMEM;
  }
  double* dout = dbuf + 3 * nb;
  const double pref = degeneracy / (8 * M_PI * M_PI * M_PI);
  int rc = VH_OK;
  if (cudaMemcpyAsync(dbuf, bins.data(), 3 * (size_t)nb * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess)
    rc = VH_E_CUDA;
  if (rc == VH_OK) {
    k_cooper_frye<D><<<(unsigned)nb, kThreads, 0, st>>>(el, count, dbuf, y, t_fo, pref, dout);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(out, dout, (size_t)nb * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
      rc = VH_E_CUDA;
  }
  if (cudaFreeAsync(dbuf, st) != cudaSuccess && rc == VH_OK) rc = VH_E_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess && rc == VH_OK) rc = VH_E_CUDA;
  return rc;
}

}  // namespace

extern "C" int vh_freezeout_2d_device(int nx, int ny, double dx, double dy, double tau0, double tau1, const double* t0,
                                      const double* t1, const double* u0, const double* u1, double t_fo, double* out,
                                      long long cap, long long* count, void* stream) {
  if (nx < 2 || ny < 2 || !(dx > 0) || !(dy > 0) || !(tau1 > tau0) || !t0 || !t1 || !u0 || !u1 || !count ||
      (cap > 0 && !out) || cap < 0)
    return VH_E_ARG;
  const vh_fo::Geo g = vh_fo::make_geo(nx, ny, 1, dx, dy, 0.0, tau0, tau1, t_fo, true);
  return surface<3>(g, t0, t1, u0, u1, out, cap, count, static_cast<cudaStream_t>(stream));
}

extern "C" int vh_freezeout_3d_device(int nx, int ny, int nz, double dx, double dy, double dz, double tau0,
                                      double tau1, const double* t0, const double* t1, const double* u0,
                                      const double* u1, double t_fo, double* out, long long cap, long long* count,
                                      void* stream) {
  if (nx < 2 || ny < 2 || nz < 2 || !(dx > 0) || !(dy > 0) || !(dz > 0) || !(tau1 > tau0) || !t0 || !t1 || !u0 ||
      !u1 || !count || (cap > 0 && !out) || cap < 0)
    return VH_E_ARG;
  const vh_fo::Geo g = vh_fo::make_geo(nx, ny, nz, dx, dy, dz, tau0, tau1, t_fo, false);
  return surface<4>(g, t0, t1, u0, u1, out, cap, count, static_cast<cudaStream_t>(stream));
}

extern "C" int vh_cooper_frye_2d_device(const double* elements, long long count, double t_fo, double mass,
                                        double degeneracy, const double* pt, int npt, const double* phi, int nphi,
                                        double* out, void* stream) {
  if ((count > 0 && !elements) || count < 0 || !(t_fo > 0) || !(mass >= 0) || !pt || !phi || npt < 1 || nphi < 1 ||
      !out || !vh_fo::bins_ok(mass, pt, npt, phi, nphi, false))
    return VH_E_ARG;
  return spectrum<3>(elements, count, t_fo, mass, degeneracy, 0.0, pt, npt, phi, nphi, out,
                     static_cast<cudaStream_t>(stream));
}

extern "C" int vh_cooper_frye_3d_device(const double* elements, long long count, double t_fo, double mass,
                                        double degeneracy, double y, const double* pt, int npt, const double* phi,
                                        int nphi, double* out, void* stream) {
  if ((count > 0 && !elements) || count < 0 || !(t_fo > 0) || !(mass >= 0) || !std::isfinite(y) || !pt || !phi ||
      npt < 1 || nphi < 1 || !out || !vh_fo::bins_ok(mass, pt, npt, phi, nphi, true))
    return VH_E_ARG;
  return spectrum<4>(elements, count, t_fo, mass, degeneracy, y, pt, npt, phi, nphi, out,
                     static_cast<cudaStream_t>(stream));
}
