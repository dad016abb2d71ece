// Operator-level kernels on a context's mesh (include/xcal.h, "operator
// level"): generic assembly of a user-built model equation, SpMV, the DILU
// preconditioner and the Green-Gauss gradient.  FP64, one row (cell) or face
// per thread, the same row routines and operation order as the persistent
// program (xcal_device.cuh), so results equal the CPU oracle bit for bit.
#include <cuda_runtime.h>

#include "xcal_device.cuh"
#include "xcal_ops.h"

namespace xcal {

namespace {

// _discretise! (Discretise_2_generated_distretisation.jl:5-81) with the terms in
// model order per face (scheme!, Discretise_1_schemes.jl:11-113), then the
// per-cell sources (scheme_source!, generated source block), then, with bcs,
// _apply_boundary_conditions! (Discretise_4_apply_bcs.jl:7-44) for the cell's
// boundary faces in condition order (functors, Discretise_3_boundary_conditions.jl).
__global__ void __launch_bounds__(TPB) assemble_terms_kernel(const __grid_constant__ KParams P,
                                                             const OpTerm *__restrict__ terms, int nterms,
                                                             const OpSource *__restrict__ srcs, int nsrc,
                                                             FieldBC bc, int use_bc, int comp,
                                                             const double *__restrict__ phi,
                                                             const double *__restrict__ prev, double dt,
                                                             double *val, double *b) {
  const int i = blockIdx.x * TPB + threadIdx.x;
  if (i >= P.n) return;
  double acc = 0.0;
  for (int k = 0; k < P.Wf; ++k) {
    const size_t e = (size_t)k * P.np + i;
    const int f = __ldg(P.f_face + e);
    if (f < 0) break;
    const double ns = (double)__ldg(P.f_sign + e);
    const int pos = __ldg(P.f_pos + e);
    double ent = __ldg(P.f_first + e) ? 0.0 : val[pos];
    for (int t = 0; t < nterms; ++t) {
      const OpTerm T = terms[t];
      if (T.kind == TERM_LAPLACIAN) {
        const double ap = T.sign * (-T.flux[f] * __ldg(P.area + f)) / __ldg(P.delta + f);
        acc += ap;
        ent += -ap;
      } else if (T.kind == TERM_DIVERGENCE && T.scheme == DIV_LINEAR) {
        const int nb = __ldg(P.f_nbr + e);
        const double ax = __ldg(P.fcx + f) - __ldg(P.ccx + i), ay = __ldg(P.fcy + f) - __ldg(P.ccy + i),
                     az = __ldg(P.fcz + f) - __ldg(P.ccz + i);
        const double bx = __ldg(P.ccx + nb) - __ldg(P.ccx + i), by = __ldg(P.ccy + nb) - __ldg(P.ccy + i),
                     bz = __ldg(P.ccz + nb) - __ldg(P.ccz + i);
        const double weight = sqrt((ax * ax + ay * ay) + az * az) / sqrt((bx * bx + by * by) + bz * bz);
        const double omw = 1.0 - weight;
        const double ap = T.sign * (T.flux[f] * ns);
        acc += ap * omw;
        ent += ap * weight;
      } else if (T.kind == TERM_DIVERGENCE) {
        const double ap = T.sign * (T.flux[f] * ns);
        acc += jmax(ap, 0.0);
        ent += -jmax(-ap, 0.0);
      }
    }
    val[pos] = ent;
  }
  const double vol = __ldg(P.vol + i);
  double bi = 0.0;
  for (int t = 0; t < nterms; ++t) {
    const OpTerm T = terms[t];
    if (T.kind == TERM_TIME && T.scheme == TIME_EULER) {
      const double rdt = 1 / dt;
      acc += vol * rdt;
      bi += prev[i] * vol * rdt;
    } else if (T.kind == TERM_SI) {
      const double flux = T.sign * T.flux[i] * vol;
      acc += flux;
    }
  }
  for (int q = 0; q < nsrc; ++q) bi += srcs[q].sign * srcs[q].field[i] * vol;
  if (use_bc) {
    for (int q = __ldg(bc.a_ptr + i); q < __ldg(bc.a_ptr + i + 1); ++q) {
      const int f = __ldg(bc.a_face + q);
      const BcEntry &E = bc.tab[__ldg(bc.a_bc + q)];
      const double value = E.v[comp];
      const bool wall = E.type == BC_NEUMANN || E.type == BC_KWALL || E.type == BC_OMEGAWALL;
      for (int t = 0; t < nterms; ++t) {
        const OpTerm T = terms[t];
        if (T.kind == TERM_LAPLACIAN) {
          if (E.type == BC_DIRICHLET) {
            const double flux = T.flux[f] * __ldg(P.area + f) / __ldg(P.delta + f);
            const double ap = T.sign * (-flux);
            acc += ap;
            bi += ap * value;
          }
        } else if (T.kind == TERM_DIVERGENCE && T.scheme == DIV_LINEAR) {
          if (E.type == BC_DIRICHLET) bi += T.sign * (-T.flux[f] * value);
          else if (wall) acc += T.sign * (T.flux[f]);
        } else if (T.kind == TERM_DIVERGENCE) {
          const double ap = T.sign * (T.flux[f]);
          if (E.type == BC_DIRICHLET) bi -= ap * value;
          else if (wall) acc += jmax(ap, 0.0);
        } else if (T.kind == TERM_SI && E.type == BC_OMEGAWALL) {
          const double flux = T.sign * T.flux[i];
          bi += flux * phi[i] * vol;
        }
      }
    }
  }
  val[__ldg(P.AU.dpos + i)] = acc;
  b[i] = bi;
}

// y = A x, ascending column order per row (CSC mul! as one row sees it).
__global__ void __launch_bounds__(TPB) spmv_kernel(Mat A, int n, const double *__restrict__ x, double *y) {
  const int i = blockIdx.x * TPB + threadIdx.x;
  if (i >= n) return;
  double o[1];
  spmv_row<1>(A, i, [&](int j, int) { return x[j]; }, o);
  y[i] = o[0];
}

// One forward level of DILU: pivots (update_dilu_diagonal!) then the forward
// row (and the backward step of rows without upper neighbours).
__global__ void __launch_bounds__(TPB) dilu_forward_level_kernel(Mat A, int n, const int *__restrict__ flev,
                                                                 const int *__restrict__ blev, int level,
                                                                 const double *__restrict__ r, double *y) {
  const int i = blockIdx.x * TPB + threadIdx.x;
  if (i >= n || flev[i] != level) return;
  dilu_setup_row(A, i);
  double in[1] = {r[i]}, o[1];
  dilu_fwd_row<1>(A, in, [&](int j, int) { return y[j]; }, i, blev[i], o);
  y[i] = o[0];
}

// One backward level of DILU (rows of backward level >= 1).
__global__ void __launch_bounds__(TPB) dilu_backward_level_kernel(Mat A, int n, const int *__restrict__ blev,
                                                                  int level, double *y) {
  const int i = blockIdx.x * TPB + threadIdx.x;
  if (i >= n || blev[i] != level) return;
  double o[1];
  dilu_bwd_row<1>(A, y, i, o);
  y[i] = o[0];
}

// interpolate! + correct_boundaries! of a scalar field (all faces).
__global__ void __launch_bounds__(TPB) face_values_kernel(const __grid_constant__ KParams P, FieldBC bc,
                                                          const double *__restrict__ phi, double *pf) {
  const int f = blockIdx.x * TPB + threadIdx.x;
  if (f >= P.nf) return;
  pf[f] = face_scalar(P, phi, f, bc, false);
}

// green_gauss! of the face values for each cell; grad as x, y, z arrays.
__global__ void __launch_bounds__(TPB) green_gauss_kernel(const __grid_constant__ KParams P,
                                                          const double *__restrict__ pf, double *grad) {
  const int i = blockIdx.x * TPB + threadIdx.x;
  if (i >= P.n) return;
  double g[3];
  green_gauss_row<3>(P, pf, i, g);
  for (int d = 0; d < 3; ++d) grad[(size_t)d * P.n + i] = g[d];
}

int blocks(int n) { return (n + TPB - 1) / TPB; }

}  // namespace

cudaError_t launch_assemble_terms(const KParams &P, const OpTerm *terms, int nterms, const OpSource *srcs, int nsrc,
                                  const FieldBC &bc, int use_bc, int comp, const double *phi, const double *prev,
                                  double dt, double *val, double *b, cudaStream_t stream) {
  (void)cudaGetLastError();
  assemble_terms_kernel<<<blocks(P.n), TPB, 0, stream>>>(P, terms, nterms, srcs, nsrc, bc, use_bc, comp, phi, prev,
                                                          dt, val, b);
  return cudaGetLastError();
}

cudaError_t launch_spmv(const Mat &A, int n, const double *x, double *y, cudaStream_t stream) {
  (void)cudaGetLastError();
  spmv_kernel<<<blocks(n), TPB, 0, stream>>>(A, n, x, y);
  return cudaGetLastError();
}

cudaError_t launch_dilu(const Mat &A, int n, const int *flev, const int *blev, int nfl, int nbl, const double *r,
                        double *y, cudaStream_t stream) {
  (void)cudaGetLastError();
  for (int l = 0; l < nfl; ++l) dilu_forward_level_kernel<<<blocks(n), TPB, 0, stream>>>(A, n, flev, blev, l, r, y);
  for (int l = 1; l < nbl; ++l) dilu_backward_level_kernel<<<blocks(n), TPB, 0, stream>>>(A, n, blev, l, y);
  return cudaGetLastError();
}

cudaError_t launch_grad(const KParams &P, const FieldBC &bc, const double *phi, double *pf, double *grad,
                        cudaStream_t stream) {
  (void)cudaGetLastError();
  face_values_kernel<<<blocks(P.nf), TPB, 0, stream>>>(P, bc, phi, pf);
  green_gauss_kernel<<<blocks(P.n), TPB, 0, stream>>>(P, pf, grad);
  return cudaGetLastError();
}

}  // namespace xcal
