// Device side of libxcal: data layout, barriers, canonical reductions and the
// per-phase routines of one SIMPLE/PISO iteration.  Everything runs inside one
// persistent kernel (xcal_kernel.cu); phases are separated by a grid-wide
// barrier (or a cluster / block barrier for small meshes).
//
// Arithmetic order: every floating-point expression reproduces the operation
// order of the reference function it implements (cited per routine), and the
// library is compiled with --fmad=false, so FP64 results equal the CPU oracle's
// bit for bit.  Reductions follow the canonical fixed tree (tiles of 1024
// values, 256 lanes x 4, warp shuffle-down tree, 8-way warp tree).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace xcal {

constexpr int TPB = 256;          // threads per CTA (fixed: canonical reduction lanes)
constexpr int TILE = 1024;        // values per canonical reduction tile
constexpr int MAXK = 8;           // partial-sum slots per phase
enum { SYNC_BLOCK = 0, SYNC_CLUSTER = 1, SYNC_GRID = 2 };
enum { PROG_SIMPLE = 0, PROG_PISO = 1, PROG_SOLVE = 2 };
enum { ST_OK = 0, ST_TIMEOUT = 1 };

struct Bar {
  unsigned long long count;
  int err;
  int pad;
};

struct BcEntry {
  int type;
  int pad;
  double v[3];
  double kappa, beta1, cmu, B, E;
};

// Boundary conditions of one field, device form.
struct FieldBC {
  const BcEntry *tab;   // [nbc] in @assign! order
  const int *a_ptr;     // [n+1] per-cell assembly entries, reference order
  const int *a_face;    // boundary face of each entry
  const int *a_bc;      // BC index of each entry
  const int *fbc;       // [nbf] BC applied to each boundary face by correct_boundaries! (-1: none)
};

struct Mat {
  const int *rp, *col, *diag, *tslot;
  double *val;
  double *Dpiv, *Dinv;  // DILU pivots and their inverses (or diagonal scaling)
  int precon;
};

struct KCfg {
  int solver, itmax;
  double atol, rtol;
};

// Krylov vectors, interleaved by system: v[i*NS + s]
struct KWork {
  double *x, *r, *p, *v, *s, *t, *q;
};

struct KParams {
  int n, nf, nbf, dim, ntiles, mode;
  // geometry (read-only for the kernel's lifetime)
  const double *vol, *ccx, *ccy, *ccz;
  const double *area, *delta, *wgt, *fnx, *fny, *fnz, *fcx, *fcy, *fcz;
  const int *o1, *o2;
  const int *cf_ptr, *cf_face, *cf_nbr, *cf_slot;
  const signed char *cf_sign;
  const unsigned char *cf_first;
  const int *cb_ptr, *cb_face;
  const int *flev, *blev;
  int nfl, nbl;
  const int *fl_ptr, *fl_rows, *bl_ptr, *bl_rows;
  Mat AU, AP;
  FieldBC bcU, bcP;
  // configuration
  int div, time, grad, piso_corr;
  double dt, nu, aU, aP;
  int has_pref, ref_cell;
  double pref;
  KCfg kU, kP;
  // state
  double *U, *Uz2;      // U [n*NS] interleaved; Uz2: z component kept for 2D meshes
  double *p, *gp, *bU, *bP, *H, *rD, *divH;
  double *mdot, *nueff, *rDf, *pf, *UfH;   // face fields (UfH [nf*NS])
  KWork wU, wP;
  double *part;         // [MAXK * ntiles]
  // outputs
  double *R;            // [iters * 4]
  int *kry;             // [iters * 5]
  int *done;            // iterations executed
  Bar *bar;
  // standalone solve
  double *sb;           // right-hand side
  int solve_solver;
  double solve_atol, solve_rtol;
  int solve_itmax;
  double *solve_out;    // [2]: iterations, final rNorm
};

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ double jmax(double a, double b) {
  if (a != a || b != b) return a + b;
  if (a > b) return a;
  if (b > a) return b;
  return signbit(a) ? b : a;
}

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_volatile_i32(const int *p) {
  return *(volatile const int *)p;
}

constexpr unsigned long long BARRIER_TIMEOUT_NS = 2000000000ull;   // 2 s

// Barrier over all CTAs of the launch.  The grid form spins with a wall-clock
// limit: on expiry it records ST_TIMEOUT in bar->err and every CTA returns.
struct Sync {
  Bar *bar;
  int mode;
  unsigned nb;
  unsigned long long epoch;
  int *ok;   // shared flag

  __device__ bool sync() {
    if (mode == SYNC_BLOCK) { __syncthreads(); return true; }
    if (mode == SYNC_CLUSTER) {
      __syncthreads();
      asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
      return true;
    }
    __syncthreads();
    epoch += 1;
    if (threadIdx.x == 0) {
      int good = 1;
      unsigned long long target = epoch * (unsigned long long)nb;
      __threadfence();
      unsigned long long v = atomicAdd(&bar->count, 1ull) + 1ull;
      if (v < target) {
        unsigned long long t0 = globaltimer();
        unsigned spins = 0;
        while (true) {
          if (ld_acquire_u64(&bar->count) >= target) break;
          if (ld_volatile_i32(&bar->err)) { good = 0; break; }
          if (((++spins) & 127u) == 0u && globaltimer() - t0 > BARRIER_TIMEOUT_NS) {
            atomicExch(&bar->err, ST_TIMEOUT);
            good = 0;
            break;
          }
        }
      }
      __threadfence();
      *ok = good;
    }
    __syncthreads();
    return *ok != 0;
  }
};

// ------------------------------------------------------ canonical reduction
// Reduce K values held by each of the 256 threads with the fixed tree; the
// result is returned in thread 0 (other threads get unspecified values).
template <int K>
__device__ __forceinline__ void block_tree(double (&s)[K], double *sm /* [8*K] */) {
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) s[k] = s[k] + __shfl_down_sync(0xffffffffu, s[k], off);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) sm[k * 8 + wid] = s[k];
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double v = (lane < 8) ? sm[k * 8 + lane] : 0.0;
#pragma unroll
      for (int off = 4; off >= 1; off >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, off);
      s[k] = v;
    }
  }
}

// Final sum of K partial arrays part[slot[k]*ntiles + t]; result broadcast to
// every thread of the CTA through sm_out.
template <int K>
__device__ __forceinline__ void final_sum(const double *part, const int (&slot)[K], int ntiles,
                                          double *sm, double *sm_out, double (&out)[K]) {
  double s[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double *pp = part + (size_t)slot[k] * ntiles;
    int t = threadIdx.x;
    double a = (t < ntiles) ? pp[t] : 0.0;
    for (int q = t + TPB; q < ntiles; q += TPB) a = a + pp[q];
    s[k] = a;
  }
  block_tree<K>(s, sm);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) sm_out[k] = s[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) out[k] = sm_out[k];
  __syncthreads();
}

// ------------------------------------------------------------- sparse rows
// y_i = sum_k val[k]*x[col[k]] in ascending column order from 0.0: the order of
// SparseArrays' CSC mul! (column scatter) as seen by one row.
template <int NS>
__device__ __forceinline__ void spmv_row(const Mat &A, const double *__restrict__ x, int i,
                                         double (&y)[NS]) {
#pragma unroll
  for (int d = 0; d < NS; ++d) y[d] = 0.0;
  const int b = __ldg(A.rp + i), e = __ldg(A.rp + i + 1);
  for (int k = b; k < e; ++k) {
    const double a = A.val[k];
    const int j = __ldg(A.col + k);
#pragma unroll
    for (int d = 0; d < NS; ++d) y[d] = y[d] + a * x[(size_t)j * NS + d];
  }
}

// DILU pivot of row i (update_dilu_diagonal!, preconditioners_1_DILU.jl:230-251):
// D_i = A_ii - sum_{j<i} (A_ij*A_ji)/D_j over lower neighbours in ascending j.
__device__ __forceinline__ void dilu_setup_row(const Mat &A, int i) {
  const int dg = __ldg(A.diag + i);
  double D = A.val[dg];
  for (int k = __ldg(A.rp + i); k < dg; ++k) {
    const int j = __ldg(A.col + k);
    D = D - A.val[k] * A.val[__ldg(A.tslot + k)] / A.Dpiv[j];
  }
  A.Dpiv[i] = D;
  A.Dinv[i] = 1 / D;
}

// Forward row (forward_substitution!, :253-279): o = in_i - sum_{j<i} (A_ij*out_j)*Dinv_j.
// Rows without upper neighbours finish the backward step at once (x_i = c_i*Dinv_i).
template <int NS>
__device__ __forceinline__ void dilu_fwd_row(const Mat &A, const double *in, double *out, int i,
                                             int blev_i, unsigned amask) {
  const int dg = __ldg(A.diag + i), b = __ldg(A.rp + i);
  double o[NS];
#pragma unroll
  for (int d = 0; d < NS; ++d) o[d] = in[(size_t)i * NS + d];
  for (int k = b; k < dg; ++k) {
    const int j = __ldg(A.col + k);
    const double a = A.val[k], dj = A.Dinv[j];
#pragma unroll
    for (int d = 0; d < NS; ++d) o[d] = o[d] - a * out[(size_t)j * NS + d] * dj;
  }
  if (blev_i == 0) {
    const double di = A.Dinv[i];
#pragma unroll
    for (int d = 0; d < NS; ++d) o[d] = o[d] * di;
  }
#pragma unroll
  for (int d = 0; d < NS; ++d)
    if (amask & (1u << d)) out[(size_t)i * NS + d] = o[d];
}

// Backward row (backward_substitution!, :281-308): x_i = c_i*Dinv_i, then
// x_i -= (A_ij*x_j)*Dinv_i for upper neighbours in ascending j.
template <int NS>
__device__ __forceinline__ void dilu_bwd_row(const Mat &A, double *out, int i, unsigned amask) {
  const int dg = __ldg(A.diag + i), e = __ldg(A.rp + i + 1);
  const double di = A.Dinv[i];
  double o[NS];
#pragma unroll
  for (int d = 0; d < NS; ++d) o[d] = out[(size_t)i * NS + d] * di;
  for (int k = dg + 1; k < e; ++k) {
    const int j = __ldg(A.col + k);
    const double a = A.val[k];
#pragma unroll
    for (int d = 0; d < NS; ++d) o[d] = o[d] - a * out[(size_t)j * NS + d] * di;
  }
#pragma unroll
  for (int d = 0; d < NS; ++d)
    if (amask & (1u << d)) out[(size_t)i * NS + d] = o[d];
}

// Diagonal preconditioners (Jacobi: 1/|A_ii|; NormDiagonal: 1/norm(column i)),
// preconditioners_2_functions.jl:28-57.
__device__ __forceinline__ void diag_precon_setup_row(const Mat &A, int i) {
  if (A.precon == 1) {
    A.Dinv[i] = 1 / fabs(A.val[__ldg(A.diag + i)]);
  } else if (A.precon == 2) {
    double s = 0.0;
    for (int k = __ldg(A.rp + i); k < __ldg(A.rp + i + 1); ++k) {
      const double a = A.val[__ldg(A.tslot + k)];
      s += a * a;
    }
    A.Dinv[i] = 1 / sqrt(s);
  } else {
    A.Dinv[i] = 1.0;
  }
}

}  // namespace xcal
