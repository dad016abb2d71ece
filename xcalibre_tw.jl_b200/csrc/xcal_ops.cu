// Operator-level entry points outside the persistent program.
//
// xcal_residual: residual!(R, equation, phi) (src/Solvers/Solvers_0_functions.jl:13-63),
//   R = sqrt(mean((A*x - b)^2)) / norm(b), with the SpMV in ascending column order
//   and the canonical reduction of xcal_device.cuh.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/xcal.h"
#include "xcal_device.cuh"
#include "xcal_ops.h"

namespace xcal {

// Per-tile partial sums of (A x - b)^2 and b^2 (one row per thread).
__global__ void __launch_bounds__(TPB) residual_tiles_kernel(int n, const int *__restrict__ rp,
                                                             const int *__restrict__ col,
                                                             const double *__restrict__ val,
                                                             const double *__restrict__ x,
                                                             const double *__restrict__ b, double *part,
                                                             int ntiles) {
  __shared__ double sm[8 * 2];
  const int t = blockIdx.x;
  const int i = t * TILE + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (i < n) {
    double y = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) y = y + val[k] * x[col[k]];
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
                            const double *b, double *part, double *out, cudaStream_t stream) {
  const int ntiles = (n + TILE - 1) / TILE;
  residual_tiles_kernel<<<ntiles, TPB, 0, stream>>>(n, rp, col, val, x, b, part, ntiles);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  residual_final_kernel<<<1, TPB, 0, stream>>>(n, part, ntiles, out);
  return cudaGetLastError();
}

}  // namespace xcal
