// Operator-level entry points outside the persistent program.
//
// xcal_residual: residual!(R, equation, phi) (src/Solvers/Solvers_0_functions.jl:13-63),
//   R = sqrt(mean((A*x - b)^2)) / norm(b), with the SpMV in ascending column order
//   and the canonical reduction of xcal_device.cuh.
// xcal_residual_noalloc: the same kernels for callers that must not allocate
//   device memory, with the per-tile partial sums in a fixed file-scope array.
#include <algorithm>
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "../../include/xcal.h"
#include "xcal_device.cuh"
#include "xcal_ops.h"

namespace xcal {

// Per-tile partial sums of (A x - b)^2 and b^2 (one row per thread).  The
// CHECKED form (allocation-free entry point, whose CSR arrays are device
// memory the host cannot validate) reads only inside the CSR's own bounds:
// a row range outside 0 <= rp[i] <= rp[i+1] <= rp[n] is skipped, as is an
// entry whose column is outside [0, n); either sets *bad.
template <bool CHECKED>
__global__ void __launch_bounds__(TPB) residual_tiles_kernel(int n, const int *__restrict__ rp,
                                                             const int *__restrict__ col,
                                                             const double *__restrict__ val,
                                                             const double *__restrict__ x,
                                                             const double *__restrict__ b, double *part,
                                                             int ntiles, int *bad) {
  __shared__ double sm[8 * 2];
  const int t = blockIdx.x;
  const int i = t * TILE + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (i < n) {
    double y = 0.0;
    int k0 = rp[i], k1 = rp[i + 1];
    if (CHECKED) {
      const int nnz = rp[n];
      if (k0 < 0 || k1 < k0 || k1 > nnz) {
        atomicOr(bad, 1);
        k1 = k0;
      }
    }
    for (int k = k0; k < k1; ++k) {
      const int j = col[k];
      if (CHECKED && (j < 0 || j >= n)) {
        atomicOr(bad, 2);
        continue;
      }
      y = y + val[k] * x[j];
    }
    const double bi = b[i];
    const double df = y - bi;
    v[0] = df * df;
    v[1] = bi * bi;
  }
  block_tree<2>(v, sm);
  if (threadIdx.x == 0) {
    part[t] = v[0];
    part[ntiles + t] = v[1];
  }
}

__global__ void __launch_bounds__(TPB) residual_final_kernel(int n, const double *part, int ntiles, double *out) {
  __shared__ double sm[8 * 2];
  __shared__ double so[2];
  double r[2];
  final_sum<2>(part, ntiles, sm, so, r);
  if (threadIdx.x == 0) out[0] = sqrt(r[0] / (double)n) / sqrt(r[1]);
}

cudaError_t launch_residual(int n, const int *rp, const int *col, const double *val, const double *x,
                            const double *b, double *part, double *out, cudaStream_t stream, int *bad) {
  const int ntiles = (n + TILE - 1) / TILE;
  (void)cudaGetLastError();   // report this launch's error, not an earlier call's
  if (bad)
    residual_tiles_kernel<true><<<ntiles, TPB, 0, stream>>>(n, rp, col, val, x, b, part, ntiles, bad);
  else
    residual_tiles_kernel<false><<<ntiles, TPB, 0, stream>>>(n, rp, col, val, x, b, part, ntiles, nullptr);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  residual_final_kernel<<<1, TPB, 0, stream>>>(n, part, ntiles, out);
  return cudaGetLastError();
}

// ------------------------------------------------ allocation-free variant
// Scratch of xcal_residual_noalloc: two partial sums per 256-row tile, for at
// most XCAL_NOALLOC_MAX_TILES tiles (16,777,216 rows), 1 MiB on every device
// that loads the library, kept until the process exits.  All calls share it.
constexpr int XCAL_NOALLOC_MAX_TILES = 65536;
constexpr int XCAL_NOALLOC_MAX_DEVICES = 64;
static __device__ __align__(256) double g_noalloc_partials[2 * XCAL_NOALLOC_MAX_TILES];
// input-check word of the same entry point (bit 1: bad row range, bit 2: bad column)
static __device__ __align__(256) int g_noalloc_bad;

// Device addresses of the scratch and the check word, resolved once per
// device with that device current (in host code the symbols name host-side
// stand-ins, not device memory).  A device reset after the first call on a
// device is not supported: the cached addresses would be stale.
static std::mutex g_noalloc_mu;
static double *g_noalloc_ptr[XCAL_NOALLOC_MAX_DEVICES] = {};
static int *g_noalloc_bad_ptr[XCAL_NOALLOC_MAX_DEVICES] = {};

cudaError_t noalloc_scratch(int device, double **out, int **bad) {
  if (device < 0 || device >= XCAL_NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void *p = nullptr, *q = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess) return e;
    e = cudaGetSymbolAddress(&q, g_noalloc_bad);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[device] = (double *)p;
    g_noalloc_bad_ptr[device] = (int *)q;
  }
  *out = g_noalloc_ptr[device];
  *bad = g_noalloc_bad_ptr[device];
  return cudaSuccess;
}

int noalloc_max_rows() { return XCAL_NOALLOC_MAX_TILES * TILE; }


__global__ void __launch_bounds__(TPB) field_scatter_kernel(int n, const double *__restrict__ src,
                                                            const int *__restrict__ perm, double *dst, int stride) {
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) dst[(size_t)perm[i] * stride] = src[i];
}

__global__ void __launch_bounds__(TPB) field_gather_kernel(int n, const double *src, const int *__restrict__ perm,
                                                           double *__restrict__ dst, int stride) {
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) dst[i] = src[(size_t)perm[i] * stride];
}

static int field_grid(int n) { return std::max(1, std::min((n + TPB - 1) / TPB, 148 * 8)); }

cudaError_t launch_field_scatter(int n, const double *src, const int *perm, double *dst, int stride,
                                 cudaStream_t stream) {
  (void)cudaGetLastError();   // report this launch's error, not an earlier call's
  field_scatter_kernel<<<field_grid(n), TPB, 0, stream>>>(n, src, perm, dst, stride);
  return cudaGetLastError();
}

cudaError_t launch_field_gather(int n, const double *src, const int *perm, double *dst, int stride,
                                cudaStream_t stream) {
  (void)cudaGetLastError();   // report this launch's error, not an earlier call's
  field_gather_kernel<<<field_grid(n), TPB, 0, stream>>>(n, src, perm, dst, stride);
  return cudaGetLastError();
}

}  // namespace xcal
