// Launchers of the operator-level kernels (xcal_ops.cu).
#pragma once
#include <cuda_runtime.h>

#include "xcal_device.cuh"

namespace xcal {
// Operator-level kernels (xcal_operators.cu).  A term / source of a
// user-built model equation with device pointers (xcal_term, xcal_source).
struct OpTerm {
  int kind, scheme;
  double sign;
  const double *flux;
};
struct OpSource {
  double sign;
  const double *field;
};
// Assembly into the ELL values `val` (zeroed by the caller) and b, with the
// mesh arrays of P; bc applied when use_bc.
cudaError_t launch_assemble_terms(const KParams &P, const OpTerm *terms, int nterms, const OpSource *srcs, int nsrc,
                                  const FieldBC &bc, int use_bc, int comp, const double *phi, const double *prev,
                                  double dt, double *val, double *b, cudaStream_t stream);
cudaError_t launch_spmv(const Mat &A, int n, const double *x, double *y, cudaStream_t stream);
// DILU set-up and application, level by level (levels of the pattern)
cudaError_t launch_dilu(const Mat &A, int n, const int *flev, const int *blev, int nfl, int nbl, const double *r,
                        double *y, cudaStream_t stream);
cudaError_t launch_grad(const KParams &P, const FieldBC &bc, const double *phi, double *pf, double *grad,
                        cudaStream_t stream);

// bad: null for CSR arrays validated on the host; else a device word that the
// kernel sets when the CSR reads out of its bounds (those reads are skipped)
cudaError_t launch_residual(int n, const int *rp, const int *col, const double *val, const double *x,
                            const double *b, double *part, double *out, cudaStream_t stream, int *bad = nullptr);
cudaError_t noalloc_scratch(int device, double **out, int **bad);
int noalloc_max_rows();
// Field transfer in the caller's cell order: dst[perm[i]*stride] = src[i] (scatter) and
// dst[i] = src[perm[i]*stride] (gather); base pointers already include the component offset.
cudaError_t launch_field_scatter(int n, const double *src, const int *perm, double *dst, int stride,
                                 cudaStream_t stream);
cudaError_t launch_field_gather(int n, const double *src, const int *perm, double *dst, int stride,
                                cudaStream_t stream);
}  // namespace xcal
