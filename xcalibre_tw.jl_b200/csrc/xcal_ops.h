// Launchers of the operator-level kernels (xcal_ops.cu).
#pragma once
#include <cuda_runtime.h>

namespace xcal {
cudaError_t launch_residual(int n, const int *rp, const int *col, const double *val, const double *x,
                            const double *b, double *part, double *out, cudaStream_t stream);
cudaError_t noalloc_scratch(int device, double **out);
int noalloc_max_rows();
}  // namespace xcal
