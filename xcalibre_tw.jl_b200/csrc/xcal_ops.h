// Launchers of the operator-level kernels (xcal_ops.cu).
#pragma once
#include <cuda_runtime.h>

namespace xcal {
cudaError_t launch_residual(int n, const int *rp, const int *col, const double *val, const double *x,
                            const double *b, double *part, double *out, cudaStream_t stream);
cudaError_t noalloc_scratch(int device, double **out);
int noalloc_max_rows();
// Field transfer in the caller's cell order: dst[perm[i]*stride] = src[i] (scatter) and
// dst[i] = src[perm[i]*stride] (gather); base pointers already include the component offset.
cudaError_t launch_field_scatter(int n, const double *src, const int *perm, double *dst, int stride,
                                 cudaStream_t stream);
cudaError_t launch_field_gather(int n, const double *src, const int *perm, double *dst, int stride,
                                cudaStream_t stream);
}  // namespace xcal
