// Device side of libxcal: data layout, barriers, canonical reductions and the
// per-row routines of one SIMPLE/PISO iteration.  Everything runs inside one
// persistent kernel (xcal_kernel.cu); phases are separated by a grid-wide
// barrier (or a cluster / block barrier for small meshes).
//
// Arithmetic order: every floating-point expression reproduces the operation
// order of the reference function it implements (cited per routine), and the
// library is compiled with --fmad=false, so FP64 results equal the CPU oracle's
// bit for bit.  Reductions follow the canonical fixed tree: tiles of 256 values
// (one per lane), warp shuffle-down tree, 8-way warp tree; tile partials folded
// per lane in ascending tile order, then the same tree.
//
// Layout: rows are padded to np = 256*ntiles.  The matrix is ELL: entry k of
// row i at k*np + i (ascending columns, column -1 in unused entries), so a
// warp's loads of one entry index are coalesced.  Per-cell internal-face lists
// use the same layout (face -1 in unused entries).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace xcal {

constexpr int TPB = 256;          // threads per CTA = lanes of the canonical reduction
constexpr int TILE = 256;         // rows per tile (one per thread)
constexpr int MAXK = 8;           // partial-sum slots
constexpr int WUNROLL = 8;        // matrix row width handled by the unrolled path
enum { SYNC_BLOCK = 0, SYNC_CLUSTER = 1, SYNC_GRID = 2 };
enum { PROG_SIMPLE = 0, PROG_PISO = 1, PROG_SOLVE = 2 };
enum { ST_OK = 0, ST_TIMEOUT = 1 };
// Phase classes of the per-phase timers (XCAL_PH_* in include/xcal.h, same order).
enum { PH_SETUP = 0, PH_MOM_ASM, PH_P_ASM, PH_PREC_SETUP, PH_KRY_SPMV, PH_KRY_PREC, PH_KRY_VEC, PH_RESID,
       PH_FACE, PH_GRAD, PH_UPDATE, PH_TURB, NPH };

struct Bar {
  unsigned long long count;
  int err;
  int nonfinite;   // set when a run stopped on a non-finite residual
};

struct BcEntry {
  int type;
  int pad;
  double v[3];
  double kappa, beta1, cmu, B, E;
  double ylam, c25;   // wall functions: y_plus_laminar(E, kappa) and cmu^0.25, computed on the host
};

// Boundary conditions of one field, device form.
struct FieldBC {
  const BcEntry *tab;   // [nbc] in @assign! order
  const int *a_ptr;     // [n+1] per-cell assembly entries, reference order
  const int *a_face;    // boundary face of each entry
  const int *a_bc;      // BC index of each entry
  const int *fbc;       // [nbf] BC applied to each boundary face by correct_boundaries! (-1: none)
};

// Sparse matrix in ELL form (shared pattern, own values).  T is the value
// type: double for the FP64 path, float for the Krylov side of the mixed path.
template <typename T>
struct MatT {
  const int *col;       // [W*np]
  const int *tpos;      // [W*np] position of the transposed entry
  const int *dpos;      // [np] position of the diagonal entry
  T *val;               // [W*np]
  T *Dpiv, *Dinv;       // DILU pivots and their inverses (or the diagonal scaling)
  T *fval;              // [W*np] ILU(0) factors: strict lower part L (unit diagonal), upper part U
  int precon, W, np;
};
using Mat = MatT<double>;

struct KCfg {
  int solver, itmax;
  double atol, rtol;
};

// Krylov vectors, interleaved by system: v[i*NS + s].  p, v and r have two
// buffers each (the fused phases read the old values of neighbours while
// writing new ones).
template <typename T>
struct KWorkT {
  T *x, *r[2], *p[2], *v[2], *s, *t, *q;
  // GMRES: Krylov basis V (vector k at V + k*n*NS, gmax+1 vectors), per-CTA
  // Givens scratch (NS x 4 x (gmax+1) doubles per CTA: c, s, z, column) and
  // the packed triangular factor R (NS x gmax*(gmax+1)/2, written by CTA 0).
  T *V;
  double *gws, *gR;
  int gmax;
};
using KWork = KWorkT<double>;

struct KParams {
  int n, nf, nbf, dim, ntiles, np, mode, Wf;
  // geometry (read-only for the kernel's lifetime)
  const double *vol, *ccx, *ccy, *ccz;
  const double *area, *delta, *wgt, *fnx, *fny, *fnz, *fcx, *fcy, *fcz;
  const int *o1, *o2;
  const int *f_face, *f_nbr, *f_pos;      // [Wf*np]
  const signed char *f_sign;
  const unsigned char *f_first;
  const int *cb_ptr, *cb_face;
  const int *flev, *blev;                 // [np]
  int nfl, nbl;
  int cg_fuse;     // CG: M^{-1} of a two-level DILU inside the x/r phase (2 barriers per iteration)
  int abort_nan;   // stop at the first non-finite Krylov residual norm
  double conv;     // SIMPLE stop: every residual <= conv (1e-7 in the reference)
  Mat AU, AP;
  FieldBC bcU, bcP;
  // configuration
  int div, time, grad;
  double dt, nu, aU, aP;
  int has_pref, ref_cell;
  double pref;
  KCfg kU, kP;
  // k-omega (RANSModels_kOmega.jl); k and omega reuse the pressure system's storage
  int model;
  double *k, *w, *nut, *nutf, *nueffk, *nueffw, *Dk, *Dw, *Pk, *Pw, *G;   // G [n*9] grad U
  FieldBC bcK, bcW, bcN;
  KCfg kK, kW;
  int precK, precW, divK, divW, timeK, timeW;
  double aK, aW;
  // mixed precision: FP32 copies of the matrices and FP32 Krylov vectors
  int prec;
  MatT<float> AU32, AP32;
  KWorkT<float> wU32, wP32;
  // state
  double *U, *Uz2;      // U [n*NS] interleaved; Uz2: z component kept for 2D meshes
  double *p, *gp, *bU, *bP, *H, *rD, *divH;
  double *mdot, *nueff, *rDf, *pf, *UfH;  // face fields (UfH [nf*NS])
  KWork wU, wP;
  double *part;         // [MAXK * ntiles]
  // outputs
  double *R;            // [iters * 4]
  int *kry;             // [iters * 5]
  int *done;            // iterations executed
  Bar *bar;
  // standalone solve
  double *sb;
  int solve_solver, solve_itmax;
  double solve_atol, solve_rtol;
  double *solve_out;    // [2]: iterations, final rNorm
  // per-phase timers (XCAL_FLAG_PHASE_TIMERS): CTA 0 accumulates SM cycles and
  // counts per phase class into phase[0..NPH) and phase[NPH..2NPH); null: off
  unsigned long long *phase;
  // grid barrier: wall-clock limit of a wait, and extra arrivals expected
  // beyond the launch's CTAs (0 in normal use; a test sets 1 so that the wait
  // can only end by its limit)
  unsigned long long bar_timeout_ns;
  int bar_extra;
};

// Codes of include/xcal.h used on the device.
enum { BC_DIRICHLET = 0, BC_NEUMANN = 1, BC_KWALL = 2, BC_OMEGAWALL = 3, BC_NUTWALL = 4 };
enum { DIV_LINEAR = 0, DIV_UPWIND = 1 };
enum { TIME_STEADY = 0, TIME_EULER = 1 };
enum { GRAD_ORTHOGONAL = 0, GRAD_MIDPOINT = 1 };
enum { SOLVER_CG = 0, SOLVER_BICGSTAB = 1, SOLVER_GMRES = 2 };
enum { PRECON_DILU = 0, PRECON_ILU0 = 4 };
enum { TERM_TIME = 0, TERM_LAPLACIAN = 1, TERM_DIVERGENCE = 2, TERM_SI = 3 };

// ------------------------------------------------------------------ serving
// Host <-> serving-kernel records, all in pinned host memory mapped into the
// device's address space (the host writes jobs and mail, the kernel writes
// results and state).  A case's device region (arena) is laid out as
// [copy | zero | scratch]; the CTAs given the case copy the first part from
// the host image and zero the second before the run.
struct ServeJob {
  KParams prm;                     // device pointers into the case's region
  const uint4 *src;                // host image of the copy part
  uint4 *dst;                      // start of the case's device region
  unsigned long long copy16, zero16;   // sizes of the copy and zero parts, in 16-byte units
  int iters, prog;
  unsigned *exits;                 // device word: CTAs of the group that left the job (0 between jobs)
  double *out_U, *out_p;           // results in device numbering: U [n*NS] interleaved, p [n]
  double *out_R;                   // [iters*4] residual histories (R_ux, R_uy, R_uz, R_p per iteration)
  int *out_kry;                    // [iters*5] Krylov counts
  int *out_state;                  // [4]: iterations done, barrier error, non-finite stop, finished (last)
};
struct ServeMail {                 // one per CTA of the serving grid
  unsigned long long seq;          // written last by the host: a new job for this CTA
  unsigned long long ack;          // written by the CTA when it takes the job
  ServeJob *job;
  int vbid, nblk;                  // this CTA's index in the job's group, and the group size
};
struct ServeCtl {
  unsigned shutdown;               // host: leave the serving loop once idle
  unsigned pad;
  unsigned long long heartbeat;    // host: advanced while the host side is alive
  unsigned long long idle_limit_ns;   // an idle CTA leaves after this long without a heartbeat
};

// ------------------------------------------------------------------ helpers
// Loads of arrays that do not change while a case runs (geometry, matrix
// pattern, level sets, boundary tables).  An ordinary launch uploads them
// before it starts, so they go through the read-only data path
// (ld.global.nc).  The serving kernel writes each case's arrays into its
// arena itself and reuses arena memory for later cases within the same
// launch: for it the arrays are not read-only for the kernel's lifetime, so
// its build (XCAL_SERVE_ONLY) reads them with ordinary coherent loads.
#if defined(XCAL_SERVE_ONLY)
template <class V>
__device__ __forceinline__ V ldro(const V *p) {
  return *p;
}
#else
template <class V>
__device__ __forceinline__ V ldro(const V *p) {
  return __ldg(p);
}
#endif

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

__device__ __forceinline__ int ld_volatile_i32(const int *p) { return *(volatile const int *)p; }

// Arrive: add with acquire-release semantics at GPU scope.  Release: the
// CTA's writes, ordered before it by the preceding block barrier, become
// visible with it.  Acquire: the last CTA to arrive (which does not poll)
// reads the count through the chain of earlier arrivals and so sees their
// writes.
__device__ __forceinline__ unsigned long long atom_add_acqrel_u64(unsigned long long *p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}

constexpr unsigned long long BARRIER_TIMEOUT_NS = 2000000000ull;   // 2 s (default limit)

// Barrier over all CTAs of the launch.  The grid form spins with a wall-clock
// limit: on expiry it records ST_TIMEOUT in bar->err and every CTA returns.
// A CTA that sees another's error stops waiting as well.
struct Sync {
  Bar *bar;
  int mode;
  unsigned nb;
  unsigned extra;                  // arrivals expected beyond the nb CTAs (0)
  unsigned long long timeout_ns;   // limit of one wait
  unsigned long long epoch;
  int *ok;   // shared flag

  __device__ __forceinline__ bool sync() {
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
      const unsigned long long target = epoch * (unsigned long long)nb + extra;
      const unsigned long long v = atom_add_acqrel_u64(&bar->count, 1ull) + 1ull;
      if (v < target) {
        const unsigned long long t0 = globaltimer();
        unsigned spins = 0;
        while (true) {
          if (ld_acquire_u64(&bar->count) >= target) break;
          if (((++spins) & 63u) == 0u) {
            if (ld_volatile_i32(&bar->err)) { good = 0; break; }
            if (globaltimer() - t0 > timeout_ns) {
              atomicExch(&bar->err, ST_TIMEOUT);
              good = 0;
              break;
            }
          }
        }
      }
      // the acquire (poll, or the arrive of the last CTA) orders the CTA's
      // later loads, through the block barrier below, after every arrive
      *ok = good;
    }
    __syncthreads();
    return *ok != 0;
  }
};

// ------------------------------------------------------ canonical reduction
// Reduce K values held by each of the 256 threads with the fixed tree; the
// result is valid in thread 0.
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

// Final sum of K partial arrays part[k*ntiles + t]; every thread of the CTA
// obtains the result.  Same tree as block_tree: each thread evaluates the
// 8-way stage itself from the staged warp sums, in the pairing of the
// shuffle-down tree (4, 2, 1), so no broadcast and only two block barriers
// are needed.  sm is free again once every thread has passed the next
// barrier, which any later writer of sm executes before writing.
template <int K>
__device__ __forceinline__ void final_sum(const double *part, int ntiles, double *sm, double *sm_out,
                                          double (&out)[K]) {
  (void)sm_out;
  double s[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double *pp = part + (size_t)k * ntiles;
    const int t = threadIdx.x;
    double a = (t < ntiles) ? pp[t] : 0.0;
    for (int q = t + TPB; q < ntiles; q += TPB) a = a + pp[q];
    s[k] = a;
  }
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
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double *w = sm + k * 8;
    double a0 = w[0] + w[4], a1 = w[1] + w[5];
    const double a2 = w[2] + w[6], a3 = w[3] + w[7];
    a0 = a0 + a2;
    a1 = a1 + a3;
    out[k] = a0 + a1;
  }
}

// ------------------------------------------------------ Krylov arithmetic
// a + s*b for Krylov vectors with a scalar s from an FP64 reduction,
// evaluated in FP64 and rounded once to the vector type.  (FP32 arithmetic
// for these updates and fused multiply-adds in the FP32 row sums were
// measured on the 128^3 cavity: at most 3 % faster, and the mixed fields
// drifted further from FP64, up to 2.7e-6 in p after 100 iterations against
// 7.5e-7.)
template <typename T>
__device__ __forceinline__ T vaxpy(T a, double s, T b) {
  return (T)((double)a + s * (double)b);
}

// ------------------------------------------------------------- sparse rows
// Row entries: all column indices of a row are loaded up front (independent,
// coalesced); the sums then run in ascending column order.
struct Row {
  int c[WUNROLL];
};
template <typename T>
__device__ __forceinline__ void load_row(const MatT<T> &A, int i, Row &r) {
#pragma unroll
  for (int k = 0; k < WUNROLL; ++k) r.c[k] = (k < A.W) ? ldro(A.col + (size_t)k * A.np + i) : -1;
}

// Row routines keep their loads out of data-dependent branches: a padding
// entry (column -1) or an entry the sum skips reads the row's own values
// instead (always in bounds), and entries past the row width re-read the last
// entry, so every entry's loads are unconditional and the scheduler may issue
// those of later entries before the sums of earlier ones.  The sums keep the
// ascending column order and skip the same entries (by selecting the old
// partial sum), so the arithmetic is unchanged.

// y = sum_k val[k]*x[col[k]] in ascending column order from 0: the order of
// SparseArrays' CSC mul! (column scatter) as seen by one row.  GetX(j, d)
// returns component d of x at row j (it may compute the value on the fly).
template <int NS, typename T, class GetX>
__device__ __forceinline__ void spmv_row(const MatT<T> &A, int i, GetX getx, T (&y)[NS]) {
#pragma unroll
  for (int d = 0; d < NS; ++d) y[d] = T(0);
  if (A.W <= WUNROLL) {
    Row r;
    load_row(A, i, r);
#pragma unroll
    for (int k = 0; k < WUNROLL; ++k) {
      const int kk = k < A.W ? k : A.W - 1;
      const int c = r.c[k];
      const int j = c >= 0 ? c : i;
      const T a = A.val[(size_t)kk * A.np + i];
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const T t = y[d] + a * getx(j, d);
        y[d] = (c >= 0) ? t : y[d];
      }
    }
  } else {
    for (int k = 0; k < A.W; ++k) {
      const int j = ldro(A.col + (size_t)k * A.np + i);
      if (j < 0) continue;
      const T a = A.val[(size_t)k * A.np + i];
#pragma unroll
      for (int d = 0; d < NS; ++d) y[d] = y[d] + a * getx(j, d);
    }
  }
}

// DILU pivot of row i (update_dilu_diagonal!, preconditioners_1_DILU.jl:230-251):
// D_i = A_ii - sum_{j<i} (A_ij*A_ji)/D_j over lower neighbours in ascending j.
template <typename T>
__device__ __forceinline__ void dilu_setup_row(const MatT<T> &A, int i) {
  T D = A.val[ldro(A.dpos + i)];
  if (A.W <= WUNROLL) {
    // Row entries are in ascending column order, so the lower neighbours are
    // the entries with 0 <= j < i.
    Row r;
    load_row(A, i, r);
#pragma unroll
    for (int k = 0; k < WUNROLL; ++k) {
      const int kk = k < A.W ? k : A.W - 1;
      const size_t e = (size_t)kk * A.np + i;
      const int c = r.c[k];
      const bool use = c >= 0 && c < i;
      const int tp = ldro(A.tpos + e);
      const int j = use ? c : i;
      const T t = D - A.val[e] * A.val[use ? tp : (int)e] / A.Dpiv[j];
      D = use ? t : D;
    }
  } else {
    for (int k = 0; k < A.W; ++k) {
      const size_t e = (size_t)k * A.np + i;
      const int j = ldro(A.col + e);
      if (j < 0 || j >= i) break;
      D = D - A.val[e] * A.val[ldro(A.tpos + e)] / A.Dpiv[j];
    }
  }
  A.Dpiv[i] = D;
  A.Dinv[i] = T(1) / D;
}

// Forward row (forward_substitution!, :253-279): o = in_i - sum_{j<i} (A_ij*out_j)*Dinv_j.
// GetOut(j, d) returns out_j (possibly recomputed); rows without upper
// neighbours also take the backward step at once (x_i = c_i*Dinv_i).
template <int NS, typename T, class GetOut>
__device__ __forceinline__ void dilu_fwd_row(const MatT<T> &A, const T (&in)[NS], GetOut geto, int i,
                                             int blev_i, T (&o)[NS]) {
#pragma unroll
  for (int d = 0; d < NS; ++d) o[d] = in[d];
  if (A.W <= WUNROLL) {
    Row r;
    load_row(A, i, r);
#pragma unroll
    for (int k = 0; k < WUNROLL; ++k) {
      const int kk = k < A.W ? k : A.W - 1;
      const int c = r.c[k];
      const bool use = c >= 0 && c < i;
      const int j = use ? c : i;
      const T a = A.val[(size_t)kk * A.np + i], dj = A.Dinv[j];
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const T t = o[d] - a * geto(j, d) * dj;
        o[d] = use ? t : o[d];
      }
    }
  } else {
    for (int k = 0; k < A.W; ++k) {
      const size_t e = (size_t)k * A.np + i;
      const int j = ldro(A.col + e);
      if (j < 0 || j >= i) break;
      const T a = A.val[e], dj = A.Dinv[j];
#pragma unroll
      for (int d = 0; d < NS; ++d) o[d] = o[d] - a * geto(j, d) * dj;
    }
  }
  if (blev_i == 0) {
    const T di = A.Dinv[i];
#pragma unroll
    for (int d = 0; d < NS; ++d) o[d] = o[d] * di;
  }
}

// Backward row (backward_substitution!, :281-308): x_i = c_i*Dinv_i, then
// x_i -= (A_ij*x_j)*Dinv_i for upper neighbours in ascending j.
template <int NS, typename T, class GetOut>
__device__ __forceinline__ void dilu_bwd_row_g(const MatT<T> &A, const T (&out_i)[NS], GetOut geto, int i,
                                               T (&o)[NS]) {
  const T di = A.Dinv[i];
#pragma unroll
  for (int d = 0; d < NS; ++d) o[d] = out_i[d] * di;
  if (A.W <= WUNROLL) {
    Row r;
    load_row(A, i, r);
#pragma unroll
    for (int k = 0; k < WUNROLL; ++k) {
      const int kk = k < A.W ? k : A.W - 1;
      const int c = r.c[k];
      const bool use = c > i;
      const int j = use ? c : i;
      const T a = A.val[(size_t)kk * A.np + i];
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const T t = o[d] - a * geto(j, d) * di;
        o[d] = use ? t : o[d];
      }
    }
  } else {
    for (int k = 0; k < A.W; ++k) {
      const size_t e = (size_t)k * A.np + i;
      const int j = ldro(A.col + e);
      if (j <= i) continue;
      const T a = A.val[e];
#pragma unroll
      for (int d = 0; d < NS; ++d) o[d] = o[d] - a * geto(j, d) * di;
    }
  }
}

// R rows at once (R > 1: the FP32 Krylov phases): the same per-row arithmetic
// as the single-row routines above, with the loads of all R rows issued
// together.  Rows of a width above WUNROLL use the single-row routines.
template <int R, int NS, typename T, class GetX>
__device__ __forceinline__ void spmv_rows(const MatT<T> &A, const int (&ii)[R], GetX getx, T (&y)[R][NS]) {
  if (A.W > WUNROLL) {
#pragma unroll
    for (int r = 0; r < R; ++r) spmv_row<NS>(A, ii[r], getx, y[r]);
    return;
  }
  Row rw[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    load_row(A, ii[r], rw[r]);
#pragma unroll
    for (int d = 0; d < NS; ++d) y[r][d] = T(0);
  }
#pragma unroll
  for (int k = 0; k < WUNROLL; ++k) {
    const int kk = k < A.W ? k : A.W - 1;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int c = rw[r].c[k];
      const int j = c >= 0 ? c : ii[r];
      const T a = A.val[(size_t)kk * A.np + ii[r]];
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const T t = y[r][d] + a * getx(j, d);
        y[r][d] = (c >= 0) ? t : y[r][d];
      }
    }
  }
}

template <int R, int NS, typename T, class GetOut>
__device__ __forceinline__ void dilu_fwd_rows(const MatT<T> &A, const T (&in)[R][NS], GetOut geto, const int (&ii)[R],
                                              const int (&bl)[R], T (&o)[R][NS]) {
  if (A.W > WUNROLL) {
#pragma unroll
    for (int r = 0; r < R; ++r) dilu_fwd_row<NS>(A, in[r], geto, ii[r], bl[r], o[r]);
    return;
  }
  Row rw[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    load_row(A, ii[r], rw[r]);
#pragma unroll
    for (int d = 0; d < NS; ++d) o[r][d] = in[r][d];
  }
#pragma unroll
  for (int k = 0; k < WUNROLL; ++k) {
    const int kk = k < A.W ? k : A.W - 1;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = ii[r], c = rw[r].c[k];
      const bool use = c >= 0 && c < i;
      const int j = use ? c : i;
      const T a = A.val[(size_t)kk * A.np + i], dj = A.Dinv[j];
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const T t = o[r][d] - a * geto(j, d) * dj;
        o[r][d] = use ? t : o[r][d];
      }
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r)
    if (bl[r] == 0) {
      const T di = A.Dinv[ii[r]];
#pragma unroll
      for (int d = 0; d < NS; ++d) o[r][d] = o[r][d] * di;
    }
}

template <int R, int NS, typename T>
__device__ __forceinline__ void dilu_bwd_rows(const MatT<T> &A, const T *out, const int (&ii)[R], T (&o)[R][NS]) {
  if (A.W > WUNROLL) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      T oi[NS];
#pragma unroll
      for (int d = 0; d < NS; ++d) oi[d] = out[(size_t)ii[r] * NS + d];
      dilu_bwd_row_g<NS>(A, oi, [&](int j, int d) { return out[(size_t)j * NS + d]; }, ii[r], o[r]);
    }
    return;
  }
  Row rw[R];
  T di[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    load_row(A, ii[r], rw[r]);
    di[r] = A.Dinv[ii[r]];
#pragma unroll
    for (int d = 0; d < NS; ++d) o[r][d] = out[(size_t)ii[r] * NS + d] * di[r];
  }
#pragma unroll
  for (int k = 0; k < WUNROLL; ++k) {
    const int kk = k < A.W ? k : A.W - 1;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = ii[r], c = rw[r].c[k];
      const bool use = c > i;
      const int j = use ? c : i;
      const T a = A.val[(size_t)kk * A.np + i];
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const T t = o[r][d] - a * out[(size_t)j * NS + d] * di[r];
        o[r][d] = use ? t : o[r][d];
      }
    }
  }
}

template <int NS, typename T>
__device__ __forceinline__ void dilu_bwd_row(const MatT<T> &A, const T *out, int i, T (&o)[NS]) {
  T oi[NS];
#pragma unroll
  for (int d = 0; d < NS; ++d) oi[d] = out[(size_t)i * NS + d];
  dilu_bwd_row_g<NS>(A, oi, [&](int j, int d) { return out[(size_t)j * NS + d]; }, i, o);
}

// ILU(0) (ILUZero.jl 0.2.0, preconditioners_0_types.jl:44-52 and
// preconditioners_2_functions.jl:59-65; the package is not vendored, so this
// restates the published algorithm).  Factor row i in level order (rows k < i
// are final): F_i = A_i, then for each lower entry k in ascending column order
// l_ik = F_ik * (1/F_kk) and F_ij -= l_ik * F_kj for every later entry j of
// row i present in row k.  Apply: y = L^{-1} v with unit diagonal (ascending
// k), then x_i = (y_i - sum_{j>i} F_ij x_j) / F_ii with the sum taken in
// descending j (the column-oriented backward sweep).
template <typename T>
__device__ __forceinline__ T ell_find(const MatT<T> &A, const T *vals, int row, int colj) {
  for (int k = 0; k < A.W; ++k) {
    const int c = ldro(A.col + (size_t)k * A.np + row);
    if (c == colj) return vals[(size_t)k * A.np + row];
    if (c < 0 || c > colj) break;
  }
  return T(0);
}
template <typename T>
__device__ __forceinline__ bool ell_has(const MatT<T> &A, int row, int colj) {
  for (int k = 0; k < A.W; ++k) {
    const int c = ldro(A.col + (size_t)k * A.np + row);
    if (c == colj) return true;
    if (c < 0 || c > colj) break;
  }
  return false;
}

template <typename T>
__device__ __forceinline__ void ilu_setup_row(const MatT<T> &A, int i) {
  for (int k = 0; k < A.W; ++k) {
    const size_t e = (size_t)k * A.np + i;
    A.fval[e] = A.val[e];
  }
  for (int k = 0; k < A.W; ++k) {
    const size_t e = (size_t)k * A.np + i;
    const int kk = ldro(A.col + e);
    if (kk < 0 || kk >= i) break;
    const T ukk = A.fval[ldro(A.dpos + kk)];
    const T l = A.fval[e] * (T(1) / ukk);
    A.fval[e] = l;
    for (int m = k + 1; m < A.W; ++m) {
      const size_t em = (size_t)m * A.np + i;
      const int j = ldro(A.col + em);
      if (j < 0) break;
      if (ell_has(A, kk, j)) A.fval[em] = A.fval[em] - l * ell_find(A, (const T *)A.fval, kk, j);
    }
  }
}

template <int NS, typename T, class GetOut>
__device__ __forceinline__ void ilu_fwd_row(const MatT<T> &A, const T (&in)[NS], GetOut geto, int i, int blev_i,
                                            T (&o)[NS]) {
#pragma unroll
  for (int d = 0; d < NS; ++d) o[d] = in[d];
  for (int k = 0; k < A.W; ++k) {
    const size_t e = (size_t)k * A.np + i;
    const int j = ldro(A.col + e);
    if (j < 0 || j >= i) break;
    const T l = A.fval[e];
#pragma unroll
    for (int d = 0; d < NS; ++d) o[d] = o[d] - l * geto(j, d);
  }
  if (blev_i == 0) {
    const T u = A.fval[ldro(A.dpos + i)];
#pragma unroll
    for (int d = 0; d < NS; ++d) o[d] = o[d] / u;
  }
}

template <int NS, typename T, class GetOut>
__device__ __forceinline__ void ilu_bwd_row_g(const MatT<T> &A, const T (&out_i)[NS], GetOut geto, int i,
                                              T (&o)[NS]) {
#pragma unroll
  for (int d = 0; d < NS; ++d) o[d] = out_i[d];
  for (int k = A.W - 1; k >= 0; --k) {
    const size_t e = (size_t)k * A.np + i;
    const int j = ldro(A.col + e);
    if (j <= i) continue;
    const T u = A.fval[e];
#pragma unroll
    for (int d = 0; d < NS; ++d) o[d] = o[d] - u * geto(j, d);
  }
  const T u = A.fval[ldro(A.dpos + i)];
#pragma unroll
  for (int d = 0; d < NS; ++d) o[d] = o[d] / u;
}

// Diagonal preconditioners (Jacobi: 1/|A_ii|; NormDiagonal: 1/norm(column i)),
// preconditioners_2_functions.jl:28-57.
template <typename T>
__device__ __forceinline__ void diag_precon_setup_row(const MatT<T> &A, int i) {
  if (A.precon == 1) {
    A.Dinv[i] = T(1) / fabs(A.val[ldro(A.dpos + i)]);
  } else if (A.precon == 2) {
    T s = T(0);
    for (int k = 0; k < A.W; ++k) {
      const size_t e = (size_t)k * A.np + i;
      if (ldro(A.col + e) < 0) continue;
      const T a = A.val[ldro(A.tpos + e)];
      s += a * a;
    }
    A.Dinv[i] = T(1) / sqrt(s);
  } else {
    A.Dinv[i] = T(1);
  }
}

// ---------------------------------------------------------- face fields
// interpolate! (Calculate_2_interpolation.jl:112-148) plus correct_boundaries!
// (:6-110) of a scalar cell field at face f.
__device__ __forceinline__ double face_scalar(const KParams &P, const double *cellv, int f, const FieldBC &bc,
                                              bool midpoint) {
  const int a = ldro(P.o1 + f), b = ldro(P.o2 + f);
  double v;
  if (midpoint) {
    v = 0.5 * (cellv[a] + cellv[b]);
  } else {
    const double w = ldro(P.wgt + f);
    const double omw = 1.0 - w;
    v = w * cellv[a] + omw * cellv[b];
  }
  if (f < P.nbf) {
    const int bi = ldro(bc.fbc + f);
    if (bi >= 0) {
      const BcEntry &e = bc.tab[bi];
      v = (e.type == BC_DIRICHLET) ? e.v[0] : cellv[a];
    }
  }
  return v;
}

// green_gauss! (Calculate_1_green_gauss.jl:2-39) of the face field pf for cell i.
template <int NS>
__device__ __forceinline__ void green_gauss_row(const KParams &P, const double *pf, int i, double (&g)[NS]) {
  double r[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k < P.Wf; ++k) {
    const size_t e = (size_t)k * P.np + i;
    const int f = ldro(P.f_face + e);
    if (f < 0) break;
    const double ns = (double)ldro(P.f_sign + e);
    const double a = ldro(P.area + f), v = pf[f];
    r[0] += v * ((a * ldro(P.fnx + f)) * ns);
    r[1] += v * ((a * ldro(P.fny + f)) * ns);
    if (NS == 3) r[2] += v * ((a * ldro(P.fnz + f)) * ns);
  }
  const double vol = ldro(P.vol + i);
#pragma unroll
  for (int d = 0; d < NS; ++d) r[d] /= vol;
  for (int q = ldro(P.cb_ptr + i); q < ldro(P.cb_ptr + i + 1); ++q) {
    const int f = ldro(P.cb_face + q);
    const double a = ldro(P.area + f), v = pf[f];
    double bx = v * (a * ldro(P.fnx + f)), by = v * (a * ldro(P.fny + f));
    bx /= vol;
    by /= vol;
    r[0] += bx;
    r[1] += by;
    if (NS == 3) {
      double bz = v * (a * ldro(P.fnz + f));
      bz /= vol;
      r[2] += bz;
    }
  }
#pragma unroll
  for (int d = 0; d < NS; ++d) g[d] = r[d];
}

}  // namespace xcal
