// The persistent device program of libxcal: one launch runs `iters` SIMPLE (or
// PISO) iterations, or one standalone Krylov solve.  Phases are separated by
// xcal::Sync barriers; every phase is "tile owned" (tile t of 256 rows is always
// processed by CTA t mod the CTA count), so a CTA may reduce over its tiles at
// the end of a phase sequence without another barrier.  Reference functions are
// cited at each phase; xcal_device.cuh states the arithmetic contract.
//
// A case runs on a group of CTAs numbered 0..vnb()-1 (vbid()): the whole grid
// of an ordinary launch, or the CTAs the serving kernel (bottom of this file)
// gives the case.
#include "xcal_device.cuh"
#include "xcal_kernel.h"

namespace xcal {

namespace {

// CTA index within the group running the case, and the group's size.
__shared__ int s_vbid, s_vnb;
__device__ __forceinline__ int vbid() { return s_vbid; }
__device__ __forceinline__ int vnb() { return s_vnb; }


// Level-scheduled preconditioners (forward and backward sweeps): DILU, ILU(0).
template <typename T>
__device__ __forceinline__ bool leveled(const MatT<T> &A) {
  return A.precon == PRECON_DILU || A.precon == PRECON_ILU0;
}
template <typename T>
__device__ __forceinline__ void lev_setup_row(const MatT<T> &A, int i) {
  if (A.precon == PRECON_ILU0) ilu_setup_row(A, i);
  else dilu_setup_row(A, i);
}
template <int NS, typename T, class GetOut>
__device__ __forceinline__ void lev_fwd_row(const MatT<T> &A, const T (&in)[NS], GetOut geto, int i, int blev_i,
                                            T (&o)[NS]) {
  if (A.precon == PRECON_ILU0) ilu_fwd_row<NS>(A, in, geto, i, blev_i, o);
  else dilu_fwd_row<NS>(A, in, geto, i, blev_i, o);
}
template <int NS, typename T>
__device__ __forceinline__ void lev_bwd_row(const MatT<T> &A, const T *out, int i, T (&o)[NS]) {
  T oi[NS];
#pragma unroll
  for (int d = 0; d < NS; ++d) oi[d] = out[(size_t)i * NS + d];
  auto g = [&](int j, int d) { return out[(size_t)j * NS + d]; };
  if (A.precon == PRECON_ILU0) ilu_bwd_row_g<NS>(A, oi, g, i, o);
  else dilu_bwd_row_g<NS>(A, oi, g, i, o);
}

constexpr int MAXTL = 32;   // tiles per CTA whose warp sums are staged in shared memory

struct Ctx {
  const KParams *P;
  Sync S;
  // Per-tile partial sums, two buffers of MAXK*ntiles used in turn by
  // successive reducing phases.  A CTA reads a reduction's partials after the
  // barrier that ends its phase while faster CTAs may already be writing the
  // next reduction's partials; with a single buffer that write could land
  // before the read.  The next write to the same buffer comes two reducing
  // phases later, behind a barrier every CTA reaches only after its read.
  double *part;
  int pw;   // buffer the next reducing phase writes
  __device__ __forceinline__ double *part_w() const { return part + (size_t)pw * MAXK * P->ntiles; }
  __device__ __forceinline__ const double *part_r() const { return part + (size_t)(pw ^ 1) * MAXK * P->ntiles; }
  double *sm;       // [8*MAXK]
  double *sm_out;   // [MAXK]
  double *ws;       // [MAXTL*MAXK*8] staged warp sums
  // per-phase timers: thread 0 of CTA 0 charges the SM cycles between two
  // barrier exits to the phase class that was current at the second one
  bool timers;
  int tag;
  long long t_last;
  unsigned long long *pacc;   // shared [2*NPH]: cycles, counts
  // Traversal direction of the tile loops, reversed at every barrier: a phase
  // then starts on the tiles the previous phase touched last, whose data are
  // the most likely still in L2 when the working set is larger than L2.  Every
  // row's values are independent of the order, so results are unchanged.
  int rev;
  __device__ __forceinline__ void phase(int t) { tag = t; }
  __device__ __forceinline__ bool sync() {
    rev ^= 1;
    const bool ok = S.sync();
    if (timers) {
      const long long t = clock64();
      pacc[tag] += (unsigned long long)(t - t_last);
      pacc[NPH + tag] += 1ull;
      t_last = t;
    }
    return ok;
  }
};

template <typename T>
__device__ __forceinline__ const MatT<T> &matU(const KParams &P) {
  if constexpr (sizeof(T) == 4) return P.AU32; else return P.AU;
}
template <typename T>
__device__ __forceinline__ const MatT<T> &matP(const KParams &P) {
  if constexpr (sizeof(T) == 4) return P.AP32; else return P.AP;
}
template <typename T>
__device__ __forceinline__ const KWorkT<T> &workU(const KParams &P) {
  if constexpr (sizeof(T) == 4) return P.wU32; else return P.wU;
}
template <typename T>
__device__ __forceinline__ const KWorkT<T> &workP(const KParams &P) {
  if constexpr (sizeof(T) == 4) return P.wP32; else return P.wP;
}

// ---------------------------------------------------------------- phases
// The CTA's tiles are vbid(), vbid() + vnb(), ...: own_tiles of them, the
// m-th in the phase's traversal direction being own_tile(m).
__device__ __forceinline__ int own_tiles(int nt) {
  const int B = vbid(), G = vnb();
  return B < nt ? (nt - 1 - B) / G + 1 : 0;
}
__device__ __forceinline__ int own_tile(int m, int cnt, int rev) {
  return vbid() + vnb() * (rev ? cnt - 1 - m : m);
}

template <class F>
__device__ __forceinline__ void tile_each(const Ctx &C, F f) {
  const KParams &P = *C.P;
  const int cnt = own_tiles(P.ntiles);
  for (int m = 0; m < cnt; ++m) {
    const int i = own_tile(m, cnt, C.rev) * TILE + threadIdx.x;
    if (i < P.n) f(i);
  }
}

// One row per thread per tile; with `reduce`, the K values returned by f are
// summed per tile with the canonical tree into part[k*ntiles + t] of the
// current partial-sum buffer (Ctx::part_w).  The warp
// stage of each tile's tree runs as the rows finish and is staged in shared
// memory; the 8-way stage of all the CTA's tiles runs once at the end, so the
// warps are not held at a block barrier per tile.
template <int K, class F>
__device__ __forceinline__ void tile_phase(Ctx &C, bool reduce, F f) {
  const KParams &P = *C.P;
  const int nt = P.ntiles, cnt = own_tiles(nt), rev = C.rev;
  if (!reduce) {
    for (int m = 0; m < cnt; ++m) {
      const int i = own_tile(m, cnt, rev) * TILE + threadIdx.x;
      double v[K];
      if (i < P.n) f(i, v);
    }
    return;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double *part = C.part_w();
  C.pw ^= 1;
  for (int m0 = 0; m0 < cnt; m0 += MAXTL) {   // chunks of at most MAXTL tiles
    const int tn = min(MAXTL, cnt - m0);
    for (int tl = 0; tl < tn; ++tl) {
      const int i = own_tile(m0 + tl, cnt, rev) * TILE + threadIdx.x;
      double v[K];
#pragma unroll
      for (int k = 0; k < K; ++k) v[k] = 0.0;
      if (i < P.n) f(i, v);
#pragma unroll
      for (int k = 0; k < K; ++k) {
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) v[k] = v[k] + __shfl_down_sync(0xffffffffu, v[k], off);
        if (lane == 0) C.ws[(tl * K + k) * 8 + wid] = v[k];
      }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < tn * K; q += TPB) {
      const double *w = C.ws + q * 8;
      double a0 = w[0] + w[4], a1 = w[1] + w[5];
      const double a2 = w[2] + w[6], a3 = w[3] + w[7];
      a0 = a0 + a2;
      a1 = a1 + a3;
      a0 = a0 + a1;
      const int k = q % K, t = own_tile(m0 + q / K, cnt, rev);
      part[(size_t)k * nt + t] = a0;
    }
    __syncthreads();
  }
}

// Rows per thread in the CG phases.  The phases are memory-latency bound (a
// row is a chain of dependent loads: columns, then neighbour values), so a
// thread keeps the loads of two rows in flight; the per-row arithmetic is
// that of the one-row routines.  128^3 cavity: FP64 22.6 -> 21.2 ms per
// SIMPLE iteration with two rows (preconditioner phases 62 -> 56 us).
template <typename T>
struct CgRows {
  static constexpr int R = 2;
};
// Row pairs pay when the CTAs hold two tiles or more each; with one tile per
// CTA or fewer (small meshes: one phase is a barrier and one row per thread)
// the one-row routines are faster.  Uniform across the CTAs of a run.
__device__ __forceinline__ bool pairs_pay(const KParams &P) { return P.ntiles >= 2 * vnb(); }

// tile_phase over R tiles at a time: the CTA takes its tiles (in the phase's
// direction) R by R, thread t row t of each (ii[r], ok[r] false past the
// mesh, where ii[r] is a valid row to read from); the per-tile reductions are
// those of tile_phase (each tile's canonical tree).
template <int K, int R, class F>
__device__ __forceinline__ void tile_phase_rows(Ctx &C, bool reduce, F f) {
  const KParams &P = *C.P;
  const int nt = P.ntiles, cnt = own_tiles(nt), rev = C.rev;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double *part = C.part_w();
  if (reduce) C.pw ^= 1;
  for (int m0 = 0; m0 < cnt; m0 += MAXTL) {
    const int tn = min(MAXTL, cnt - m0);
    for (int tl = 0; tl < tn; tl += R) {
      int ii[R];
      bool ok[R], tv[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        tv[r] = tl + r < tn;
        const int i = (tv[r] ? own_tile(m0 + tl + r, cnt, rev) : 0) * TILE + threadIdx.x;
        ok[r] = tv[r] && i < P.n;
        ii[r] = ok[r] ? i : 0;
      }
      double v[R][K];
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int k = 0; k < K; ++k) v[r][k] = 0.0;
      f(ii, ok, v);
      if (reduce)
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if (!tv[r]) continue;
#pragma unroll
          for (int k = 0; k < K; ++k) {
            double x = v[r][k];
#pragma unroll
            for (int off = 16; off >= 1; off >>= 1) x = x + __shfl_down_sync(0xffffffffu, x, off);
            if (lane == 0) C.ws[((tl + r) * K + k) * 8 + wid] = x;
          }
        }
    }
    if (!reduce) continue;
    __syncthreads();
    for (int q = threadIdx.x; q < tn * K; q += TPB) {
      const double *w = C.ws + q * 8;
      double a0 = w[0] + w[4], a1 = w[1] + w[5];
      const double a2 = w[2] + w[6], a3 = w[3] + w[7];
      a0 = a0 + a2;
      a1 = a1 + a3;
      a0 = a0 + a1;
      const int k = q % K, t = own_tile(m0 + q / K, cnt, rev);
      part[(size_t)k * nt + t] = a0;
    }
    __syncthreads();
  }
}

template <class F>
__device__ __forceinline__ void grid_each(int count, F f) {
  for (int i = vbid() * TPB + threadIdx.x; i < count; i += vnb() * TPB) f(i);
}

template <int NS>
__device__ __forceinline__ void ld(const double *a, int i, double (&o)[NS]) {
#pragma unroll
  for (int d = 0; d < NS; ++d) o[d] = a[(size_t)i * NS + d];
}
template <int NS>
__device__ __forceinline__ void st(double *a, int i, const double (&o)[NS]) {
#pragma unroll
  for (int d = 0; d < NS; ++d) a[(size_t)i * NS + d] = o[d];
}

// ------------------------------------------------------- preconditioning
// Row-local part of M^{-1}: DILU forward level 0 (and the backward step of
// rows without upper neighbours) or a diagonal scaling.  Returns false when
// the row has no row-local part (DILU rows of level >= 1).
template <int NS, typename T>
__device__ __forceinline__ bool precon_local(const KParams &P, const MatT<T> &A, int i, const T (&in)[NS],
                                             T (&o)[NS]) {
  if (A.precon == PRECON_DILU) {
    if (ldro(P.flev + i) != 0) return false;
#pragma unroll
    for (int d = 0; d < NS; ++d) o[d] = in[d];
    if (ldro(P.blev + i) == 0) {
      const T di = A.Dinv[i];
#pragma unroll
      for (int d = 0; d < NS; ++d) o[d] = o[d] * di;
    }
    return true;
  }
  if (A.precon == PRECON_ILU0) {
    if (ldro(P.flev + i) != 0) return false;
#pragma unroll
    for (int d = 0; d < NS; ++d) o[d] = in[d];
    if (ldro(P.blev + i) == 0) {
      const T u = A.fval[ldro(A.dpos + i)];
#pragma unroll
      for (int d = 0; d < NS; ++d) o[d] = o[d] / u;
    }
    return true;
  }
  const T di = A.Dinv[i];
#pragma unroll
  for (int d = 0; d < NS; ++d) o[d] = di * in[d];
  return true;
}

// Number of phases of M^{-1} after its producer phase.  The producer did the
// row-local part (and, with first_lvl == 2, forward level 1 as well).
template <typename T>
__device__ __forceinline__ int precon_tail_phases(const KParams &P, const MatT<T> &A, bool setup, int first_lvl) {
  if (!leveled(A)) return setup ? 1 : 0;
  return max(0, P.nfl - first_lvl) + (P.nbl - 1);
}

// The remaining phases of M^{-1} (in -> out).  With `setup` the DILU pivots
// (update_preconditioner!) are computed level by level in the same phases.
// The last phase also computes the K partial sums red(i, v).
template <int NS, int K, typename T, class Red, int R = 1>
__device__ __forceinline__ bool precon_tail(Ctx &C, const MatT<T> &A, const T *in, T *out, bool setup, int first_lvl, Red red) {
  const KParams &P = *C.P;
  const int nph = precon_tail_phases(P, A, setup, first_lvl);
  C.phase(setup ? PH_PREC_SETUP : PH_KRY_PREC);
  if constexpr (R > 1) {
    if (!setup && A.precon == PRECON_DILU && nph > 0 && pairs_pay(P)) {
      // the DILU levels R rows at a time; in a warp holding a row of the
      // level, rows outside it compute with what they read and store
      // nothing; a warp without one skips the rows (with a level-ordered
      // numbering whole tiles lie outside each level)
      int ph = 0;
      for (int l = first_lvl; l < P.nfl; ++l) {
        const bool last = (++ph == nph);
        tile_phase_rows<K, R>(C, last, [&](const int (&ii)[R], const bool (&ok)[R], double (&v)[R][K]) {
          bool at[R], any = false;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            at[r] = ok[r] && ldro(P.flev + ii[r]) == l;
            any = any || at[r];
          }
          if (__any_sync(0xffffffffu, any)) {
            T iv[R][NS], o[R][NS];
            int bl[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
              bl[r] = ldro(P.blev + ii[r]);
#pragma unroll
              for (int d = 0; d < NS; ++d) iv[r][d] = in[(size_t)ii[r] * NS + d];
            }
            dilu_fwd_rows<R, NS>(A, iv, [&](int j, int d) { return out[(size_t)j * NS + d]; }, ii, bl, o);
#pragma unroll
            for (int r = 0; r < R; ++r)
              if (at[r])
#pragma unroll
                for (int d = 0; d < NS; ++d) out[(size_t)ii[r] * NS + d] = o[r][d];
          }
          if (last)
#pragma unroll
            for (int r = 0; r < R; ++r)
              if (ok[r]) red(ii[r], v[r]);
        });
        if (!C.sync()) return false;
      }
      for (int l = 1; l < P.nbl; ++l) {
        const bool last = (++ph == nph);
        tile_phase_rows<K, R>(C, last, [&](const int (&ii)[R], const bool (&ok)[R], double (&v)[R][K]) {
          bool at[R], any = false;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            at[r] = ok[r] && ldro(P.blev + ii[r]) == l;
            any = any || at[r];
          }
          if (__any_sync(0xffffffffu, any)) {
            T o[R][NS];
            dilu_bwd_rows<R, NS>(A, out, ii, o);
#pragma unroll
            for (int r = 0; r < R; ++r)
              if (at[r])
#pragma unroll
                for (int d = 0; d < NS; ++d) out[(size_t)ii[r] * NS + d] = o[r][d];
          }
          if (last)
#pragma unroll
            for (int r = 0; r < R; ++r)
              if (ok[r]) red(ii[r], v[r]);
        });
        if (!C.sync()) return false;
      }
      return true;
    }
  }
  if (nph == 0 && setup) {   // nothing left to apply: reduce in a phase of its own
    tile_phase<K>(C, true, [&](int i, double (&v)[K]) { red(i, v); });
    return C.sync();
  }
  if (!leveled(A)) {
    if (!setup) return true;
    tile_phase<K>(C, true, [&](int i, double (&v)[K]) {
      diag_precon_setup_row(A, i);
      const T di = A.Dinv[i];
#pragma unroll
      for (int d = 0; d < NS; ++d) out[(size_t)i * NS + d] = di * in[(size_t)i * NS + d];
      red(i, v);
    });
    return C.sync();
  }
  int ph = 0;
  for (int l = first_lvl; l < P.nfl; ++l) {
    const bool last = (++ph == nph);
    tile_phase<K>(C, last, [&](int i, double (&v)[K]) {
      if (ldro(P.flev + i) == l) {
        if (setup) lev_setup_row(A, i);
        T iv[NS], o[NS];
#pragma unroll
        for (int d = 0; d < NS; ++d) iv[d] = in[(size_t)i * NS + d];
        lev_fwd_row<NS>(A, iv, [&](int j, int d) { return out[(size_t)j * NS + d]; }, i, ldro(P.blev + i), o);
#pragma unroll
        for (int d = 0; d < NS; ++d) out[(size_t)i * NS + d] = o[d];
      }
      if (last) red(i, v);
    });
    if (!C.sync()) return false;
  }
  for (int l = 1; l < P.nbl; ++l) {
    const bool last = (++ph == nph);
    tile_phase<K>(C, last, [&](int i, double (&v)[K]) {
      if (ldro(P.blev + i) == l) {
        T o[NS];
        lev_bwd_row<NS>(A, out, i, o);
#pragma unroll
        for (int d = 0; d < NS; ++d) out[(size_t)i * NS + d] = o[d];
      }
      if (last) red(i, v);
    });
    if (!C.sync()) return false;
  }
  return true;
}

// Krylov start for row i (Krylov.jl warm start): r0 = b - A*x0 in FP64 over
// the row just assembled, x = 0, the DILU pivot of level-0 rows and the
// row-local part of the first M^{-1}.  With T = float the row is also copied
// to the FP32 matrix the Krylov iterations use (iterative refinement: the
// FP64 residual r0 is the right-hand side of an FP32 correction solve).
// BiCGSTAB keeps r0 in q and preconditions into r[0]; CG keeps r[0] = r0 and
// preconditions into v[0].
template <int NS, typename T>
__device__ __forceinline__ void krylov_init_row(const KParams &P, const Mat &A64, const MatT<T> &A,
                                                const KWorkT<T> &w, const double (&b)[NS], const double *x0,
                                                int i, int solver) {
  if constexpr (sizeof(T) == 4) {
    // every entry, padding included (zero in the FP64 matrix)
    for (int k = 0; k < A.W; ++k) {
      const size_t e = (size_t)k * A.np + i;
      A.val[e] = (float)A64.val[e];
    }
  }
  double y[NS];
  T r0[NS];
  spmv_row<NS>(A64, i, [&](int j, int d) { return x0[(size_t)j * NS + d]; }, y);
#pragma unroll
  for (int d = 0; d < NS; ++d) {
    r0[d] = (T)(b[d] - y[d]);
    w.x[(size_t)i * NS + d] = T(0);
  }
  if (leveled(A) && ldro(P.flev + i) == 0) lev_setup_row(A, i);
  T o[NS];
  const bool dilu = leveled(A);
  if (solver != SOLVER_CG) {
#pragma unroll
    for (int d = 0; d < NS; ++d) w.q[(size_t)i * NS + d] = r0[d];
    if (dilu && precon_local<NS>(P, A, i, r0, o))
#pragma unroll
      for (int d = 0; d < NS; ++d) w.r[0][(size_t)i * NS + d] = o[d];
  } else {
#pragma unroll
    for (int d = 0; d < NS; ++d) w.r[0][(size_t)i * NS + d] = r0[d];
    if (dilu && precon_local<NS>(P, A, i, r0, o))
#pragma unroll
      for (int d = 0; d < NS; ++d) w.v[0][(size_t)i * NS + d] = o[d];
  }
}

// Set-up phases of M and its first application after the assembly phase,
// with the initial dot products (CG: <r,z>; BiCGSTAB: <b,r>, <r,r>), all
// accumulated in FP64.
template <int NS, typename T>
__device__ __forceinline__ bool krylov_start(Ctx &C, const MatT<T> &A, const KWorkT<T> &w, const double *b, int solver) {
  if (solver != SOLVER_CG) {
    return precon_tail<NS, 2 * NS>(C, A, w.q, w.r[0], true, 1, [&](int i, double (&v)[2 * NS]) {
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const double rv = (double)w.r[0][(size_t)i * NS + d];
        v[2 * d] = b[(size_t)i * NS + d] * rv;
        v[2 * d + 1] = rv * rv;
      }
    });
  }
  return precon_tail<NS, NS>(C, A, w.r[0], w.v[0], true, 1, [&](int i, double (&v)[NS]) {
#pragma unroll
    for (int d = 0; d < NS; ++d)
      v[d] = (double)w.r[0][(size_t)i * NS + d] * (double)w.v[0][(size_t)i * NS + d];
  });
}

// ------------------------------------------------------------- BiCGSTAB
// Krylov.jl 0.9.5 bicgstab! with left preconditioner M, N = I, c = b.
// Entry: r[0] = M^{-1}(b - A x0), x = 0, partials <b,r>, <r,r> in part.
// Fused phases per iteration:
//   A  p = r + beta*(p - omega*v) (recomputed for neighbours), q = A p, M^-1 level 0
//   .. remaining M^-1 phases, last one reduces <b,v>
//   D  s = r - alpha*v (recomputed for neighbours), x += alpha*p, q = A s, M^-1 level 0
//   .. remaining M^-1 phases, last one reduces <t,s>, <t,t>
//   G  x += omega*s, r = s - omega*t, reduces <b,r>, <r,r>
// Vector updates are evaluated in FP64 and stored in T; dots accumulate in FP64.
template <int NS, typename T>
__device__ __forceinline__ bool bicgstab(Ctx &C, const MatT<T> &A, const KWorkT<T> &w, const double *bb, const KCfg &cfg,
                         int (&its)[NS], double (&rnorm_out)[NS]) {
  const KParams &P = *C.P;
  double red[2 * NS];
  final_sum<2 * NS>(C.part_r(), P.ntiles, C.sm, C.sm_out, red);
  double rho[NS], alpha[NS], omega[NS], beta[NS], rnorm[NS], eps[NS], nrho[NS];
  unsigned active = 0;
#pragma unroll
  for (int d = 0; d < NS; ++d) {
    its[d] = 0;
    rnorm[d] = sqrt(red[2 * d + 1]);
    rho[d] = 1.0; alpha[d] = 1.0; omega[d] = 1.0; beta[d] = 0.0;
    eps[d] = 0.0; nrho[d] = 0.0;
    if (rnorm[d] == 0.0) continue;
    eps[d] = cfg.atol + cfg.rtol * rnorm[d];
    nrho[d] = red[2 * d];
    if (nrho[d] == 0.0) continue;
    const bool solved = rnorm[d] <= eps[d], tired = 0 >= cfg.itmax;
    if (!(solved || tired)) active |= 1u << d;
  }
  T *r = w.r[0];
  const int tail = precon_tail_phases(P, A, false, 1);
  int pc = 0;
  bool first = true;
  while (active) {
#pragma unroll
    for (int d = 0; d < NS; ++d)
      if (active & (1u << d)) { its[d] += 1; rho[d] = nrho[d]; }
    T *pn = w.p[pc], *po = w.p[pc ^ 1], *vn = w.v[pc], *vo = w.v[pc ^ 1];
    auto getp = [&](int j, int d) -> T {
      const size_t k = (size_t)j * NS + d;
      if (first) return r[k];
      const double pv = (double)po[k] + (-omega[d]) * (double)vo[k];
      return (T)((double)r[k] + beta[d] * pv);
    };
    // A: p update, q = A p, M^{-1} row-local part
    C.phase(PH_KRY_SPMV);
    tile_phase<NS>(C, tail == 0, [&](int i, double (&v)[NS]) {
      T y[NS], pi[NS], o[NS];
      spmv_row<NS>(A, i, getp, y);
#pragma unroll
      for (int d = 0; d < NS; ++d) pi[d] = getp(i, d);
#pragma unroll
      for (int d = 0; d < NS; ++d)
        if (active & (1u << d)) pn[(size_t)i * NS + d] = pi[d];
#pragma unroll
      for (int d = 0; d < NS; ++d) w.q[(size_t)i * NS + d] = y[d];
      if (precon_local<NS>(P, A, i, y, o))
#pragma unroll
        for (int d = 0; d < NS; ++d) vn[(size_t)i * NS + d] = o[d];
      if (tail == 0)
#pragma unroll
        for (int d = 0; d < NS; ++d) v[d] = bb[(size_t)i * NS + d] * (double)o[d];
    });
    if (!C.sync()) return false;
    if (!precon_tail<NS, NS>(C, A, (const T *)w.q, vn, false, 1, [&](int i, double (&v)[NS]) {
#pragma unroll
          for (int d = 0; d < NS; ++d) v[d] = bb[(size_t)i * NS + d] * (double)vn[(size_t)i * NS + d];
        }))
      return false;
    {
      double cv[NS];
      final_sum<NS>(C.part_r(), P.ntiles, C.sm, C.sm_out, cv);
#pragma unroll
      for (int d = 0; d < NS; ++d)
        if (active & (1u << d)) alpha[d] = rho[d] / cv[d];
    }
    auto gets = [&](int j, int d) -> T {
      const size_t k = (size_t)j * NS + d;
      return vaxpy<T>(r[k], -alpha[d], vn[k]);
    };
    // D: s, x += alpha p, q = A s, M^{-1} row-local part
    C.phase(PH_KRY_SPMV);
    tile_phase<2 * NS>(C, tail == 0, [&](int i, double (&v)[2 * NS]) {
      T y[NS], o[NS], si[NS];
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const size_t k = (size_t)i * NS + d;
        si[d] = gets(i, d);
        if (active & (1u << d)) {
          w.s[k] = si[d];
          w.x[k] = vaxpy<T>(w.x[k], alpha[d], pn[k]);
        }
      }
      spmv_row<NS>(A, i, gets, y);
#pragma unroll
      for (int d = 0; d < NS; ++d) w.q[(size_t)i * NS + d] = y[d];
      if (precon_local<NS>(P, A, i, y, o))
#pragma unroll
        for (int d = 0; d < NS; ++d) w.t[(size_t)i * NS + d] = o[d];
      if (tail == 0)
#pragma unroll
        for (int d = 0; d < NS; ++d) {
          v[2 * d] = (double)o[d] * (double)si[d];
          v[2 * d + 1] = (double)o[d] * (double)o[d];
        }
    });
    if (!C.sync()) return false;
    if (!precon_tail<NS, 2 * NS>(C, A, (const T *)w.q, w.t, false, 1, [&](int i, double (&v)[2 * NS]) {
#pragma unroll
          for (int d = 0; d < NS; ++d) {
            const size_t k = (size_t)i * NS + d;
            const double tv = (double)w.t[k];
            v[2 * d] = tv * (double)w.s[k];
            v[2 * d + 1] = tv * tv;
          }
        }))
      return false;
    final_sum<2 * NS>(C.part_r(), P.ntiles, C.sm, C.sm_out, red);
#pragma unroll
    for (int d = 0; d < NS; ++d)
      if (active & (1u << d)) omega[d] = red[2 * d] / red[2 * d + 1];
    // G: x += omega s, r = s - omega t, <b,r>, <r,r>
    C.phase(PH_KRY_VEC);
    tile_phase<2 * NS>(C, true, [&](int i, double (&v)[2 * NS]) {
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const size_t k = (size_t)i * NS + d;
        double rv = (double)r[k];
        if (active & (1u << d)) {
          w.x[k] = vaxpy<T>(w.x[k], omega[d], w.s[k]);
          const T rt = vaxpy<T>(w.s[k], -omega[d], w.t[k]);
          r[k] = rt;
          rv = (double)rt;
        }
        v[2 * d] = bb[k] * rv;
        v[2 * d + 1] = rv * rv;
      }
    });
    if (!C.sync()) return false;
    final_sum<2 * NS>(C.part_r(), P.ntiles, C.sm, C.sm_out, red);
    unsigned cont = 0;
#pragma unroll
    for (int d = 0; d < NS; ++d) {
      if (!(active & (1u << d))) continue;
      nrho[d] = red[2 * d];
      beta[d] = (nrho[d] / rho[d]) * (alpha[d] / omega[d]);
      rnorm[d] = sqrt(red[2 * d + 1]);
      const bool mach = (rnorm[d] + 1.0 <= 1.0);
      const bool solved = (rnorm[d] <= eps[d]) || mach;
      const bool tired = its[d] >= cfg.itmax;
      const bool breakdown = (alpha[d] == 0.0 || isnan(alpha[d]));
      if (!(solved || tired || breakdown)) cont |= 1u << d;
    }
    active = cont;
    first = false;
    pc ^= 1;
  }
#pragma unroll
  for (int d = 0; d < NS; ++d) rnorm_out[d] = rnorm[d];
  return true;
}

// ------------------------------------------------------------------- CG
// Krylov.jl 0.9.5 cg! with preconditioner M.  The sign of <r,z> at the start
// selects the formulation: for a negative definite system CG runs on (-A)x=-b,
// i.e. <r,z> and <p,Ap> enter with their sign flipped (negation is exact).
// Entry: r[0] = b - A x0, v[0] = M^{-1} r, x = 0, partial <r,z> in part.
// Fused phases per iteration:
//   A  p = z + beta*p (recomputed for neighbours), q = A p, reduces <p,q>
//   B  x += alpha p, r -= alpha q, M^-1 levels 0 and 1 (level-0 values of
//      neighbours recomputed), backward step of rows without upper neighbours
//   .. remaining M^-1 phases, the last reduces <r,z>
template <int NS, typename T>
__device__ __forceinline__ bool cg(Ctx &C, const MatT<T> &A, const KWorkT<T> &w, const KCfg &cfg, int (&its)[NS],
                   double (&rnorm_out)[NS]) {
  const KParams &P = *C.P;
  const double EPS = 2.220446049250313e-16;
  double red[NS];
  final_sum<NS>(C.part_r(), P.ntiles, C.sm, C.sm_out, red);
  double gamma[NS], sgn[NS], rnorm[NS], pn2[NS], eps[NS], alpha[NS], beta[NS];
  unsigned active = 0;
#pragma unroll
  for (int d = 0; d < NS; ++d) {
    its[d] = 0;
    sgn[d] = (red[d] < 0.0) ? -1.0 : 1.0;
    gamma[d] = sgn[d] * red[d];
    rnorm[d] = sqrt(gamma[d]);
    alpha[d] = 0.0; beta[d] = 0.0; pn2[d] = gamma[d]; eps[d] = 0.0;
    if (gamma[d] == 0.0) continue;
    eps[d] = cfg.atol + cfg.rtol * rnorm[d];
    const bool solved = rnorm[d] <= eps[d], tired = 0 >= cfg.itmax;
    if (!(solved || tired)) active |= 1u << d;
  }
  const T *z = w.v[0];
  T *zw = w.v[0];
  const bool dilu = leveled(A);
  const bool lvl1 = dilu && P.nfl >= 2;
  // With two forward levels every level-1 row has only lower neighbours and
  // every level-0 row only upper ones, so the whole of M^{-1} r fits in the
  // x/r phase: level-0 rows recompute their upper neighbours' forward values
  // (which in turn recompute r of their level-0 neighbours).  Same row
  // functions, same inputs: identical bits, one grid barrier fewer.
  const bool fuse = A.precon == PRECON_DILU && P.nfl == 2 && P.cg_fuse;
  const int tail = (dilu && !fuse) ? precon_tail_phases(P, A, false, 2) : 0;
  int rc = 0, pc = 0;
  bool first = true;
  while (active) {
    T *pn = w.p[pc], *po = w.p[pc ^ 1];
    auto getp = [&](int j, int d) -> T {
      const size_t k = (size_t)j * NS + d;
      if (first) return z[k];
      return vaxpy<T>(z[k], beta[d], po[k]);
    };
    // A: p update, q = A p, <p,q>
    C.phase(PH_KRY_SPMV);
    if (CgRows<T>::R > 1 && pairs_pay(P)) {
      constexpr int R = CgRows<T>::R;
      tile_phase_rows<NS, R>(C, true, [&](const int (&ii)[R], const bool (&ok)[R], double (&v)[R][NS]) {
        T y[R][NS];
        spmv_rows<R, NS>(A, ii, getp, y);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if (!ok[r]) continue;
          const int i = ii[r];
#pragma unroll
          for (int d = 0; d < NS; ++d) {
            const T pi = getp(i, d);
            if (active & (1u << d)) pn[(size_t)i * NS + d] = pi;
            v[r][d] = (double)pi * (double)y[r][d];
            w.q[(size_t)i * NS + d] = y[r][d];
          }
        }
      });
    } else {
      tile_phase<NS>(C, true, [&](int i, double (&v)[NS]) {
        T y[NS];
        spmv_row<NS>(A, i, getp, y);
#pragma unroll
        for (int d = 0; d < NS; ++d) {
          const T pi = getp(i, d);
          if (active & (1u << d)) pn[(size_t)i * NS + d] = pi;
          v[d] = (double)pi * (double)y[d];
          w.q[(size_t)i * NS + d] = y[d];
        }
      });
    }
    if (!C.sync()) return false;
    final_sum<NS>(C.part_r(), P.ntiles, C.sm, C.sm_out, red);
    unsigned upd = 0;
#pragma unroll
    for (int d = 0; d < NS; ++d) {
      if (!(active & (1u << d))) continue;
      const double pAp = sgn[d] * red[d];
      if (pAp <= EPS * pn2[d] && fabs(pAp) <= EPS * pn2[d]) continue;   // zero curvature: stop
      alpha[d] = gamma[d] / pAp;
      upd |= 1u << d;
    }
    active = upd;
    if (!active) break;
    T *ro = w.r[rc], *rn = w.r[rc ^ 1];
    auto getr = [&](int j, int d) -> T {
      const size_t k = (size_t)j * NS + d;
      return vaxpy<T>(ro[k], -alpha[d], w.q[k]);
    };
    // B: x, r updates and M^{-1} levels 0/1
    C.phase(PH_KRY_PREC);
    if (CgRows<T>::R > 1 && pairs_pay(P)) {
      if (A.precon == PRECON_DILU && !fuse) {
        // R rows at a time; a DILU row of level 0 or 1 is one forward row
        // (level 0: no lower neighbours, then its diagonal step when it has
        // no upper ones), the row-local part of precon_local for level 0
        constexpr int R = CgRows<T>::R;
        tile_phase_rows<NS, R>(C, tail == 0, [&](const int (&ii)[R], const bool (&ok)[R], double (&v)[R][NS]) {
          T rr[R][NS], o[R][NS];
          int fl[R], bl[R];
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int i = ii[r];
            fl[r] = ldro(P.flev + i);
            bl[r] = ldro(P.blev + i);
#pragma unroll
            for (int d = 0; d < NS; ++d) {
              const size_t k = (size_t)i * NS + d;
              rr[r][d] = getr(i, d);
              if (ok[r] && (active & (1u << d))) {
                w.x[k] = vaxpy<T>(w.x[k], alpha[d], pn[k]);
                rn[k] = rr[r][d];
              }
            }
          }
          // only level-1 rows have lower neighbours to sum over; a warp
          // without one takes the row-local step (level 0: o = r, scaled by
          // the pivot's inverse when the row has no upper neighbours)
          bool any = false;
#pragma unroll
          for (int r = 0; r < R; ++r) any = any || (ok[r] && lvl1 && fl[r] == 1);
          if (__any_sync(0xffffffffu, any)) {
            dilu_fwd_rows<R, NS>(A, rr, getr, ii, bl, o);
          } else {
#pragma unroll
            for (int r = 0; r < R; ++r) {
#pragma unroll
              for (int d = 0; d < NS; ++d) o[r][d] = rr[r][d];
              if (bl[r] == 0) {
                const T di = A.Dinv[ii[r]];
#pragma unroll
                for (int d = 0; d < NS; ++d) o[r][d] = o[r][d] * di;
              }
            }
          }
#pragma unroll
          for (int r = 0; r < R; ++r) {
            if (!ok[r]) continue;
            const bool have = fl[r] == 0 || (lvl1 && fl[r] == 1);
            if (have)
#pragma unroll
              for (int d = 0; d < NS; ++d) zw[(size_t)ii[r] * NS + d] = o[r][d];
            if (tail == 0)
#pragma unroll
              for (int d = 0; d < NS; ++d) v[r][d] = (double)rr[r][d] * (double)o[r][d];
          }
        });
        goto phase_b_done;
      }
    }
    tile_phase<NS>(C, tail == 0, [&](int i, double (&v)[NS]) {
      T rr[NS], o[NS];
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const size_t k = (size_t)i * NS + d;
        rr[d] = getr(i, d);
        if (active & (1u << d)) {
          w.x[k] = vaxpy<T>(w.x[k], alpha[d], pn[k]);
          rn[k] = rr[d];
        }
      }
      bool have;
      if (fuse) {
        if (ldro(P.flev + i) == 1) {
          dilu_fwd_row<NS>(A, rr, getr, i, 0, o);
        } else if (ldro(P.blev + i) == 0) {
#pragma unroll
          for (int d = 0; d < NS; ++d) o[d] = rr[d] * A.Dinv[i];
        } else {
          dilu_bwd_row_g<NS>(A, rr, [&](int j, int d) -> T {
            T rj[NS], zj[NS];
#pragma unroll
            for (int e = 0; e < NS; ++e) rj[e] = getr(j, e);
            dilu_fwd_row<NS>(A, rj, getr, j, 0, zj);
            return zj[d];
          }, i, o);
        }
        have = true;
      } else {
        have = precon_local<NS>(P, A, i, rr, o);
        if (!have && lvl1 && ldro(P.flev + i) == 1) {
          lev_fwd_row<NS>(A, rr, getr, i, ldro(P.blev + i), o);
          have = true;
        }
      }
      if (have)
#pragma unroll
        for (int d = 0; d < NS; ++d) zw[(size_t)i * NS + d] = o[d];
      if (tail == 0)
#pragma unroll
        for (int d = 0; d < NS; ++d) v[d] = (double)rr[d] * (double)o[d];
    });
  phase_b_done:
    if (!C.sync()) return false;
    if (dilu && !fuse) {
      auto rz = [&](int i, double (&v)[NS]) {
#pragma unroll
        for (int d = 0; d < NS; ++d) v[d] = (double)rn[(size_t)i * NS + d] * (double)z[(size_t)i * NS + d];
      };
      if (!precon_tail<NS, NS, T, decltype(rz), CgRows<T>::R>(C, A, (const T *)rn, zw, false, 2, rz)) return false;
    }
    final_sum<NS>(C.part_r(), P.ntiles, C.sm, C.sm_out, red);
    unsigned cont = 0;
#pragma unroll
    for (int d = 0; d < NS; ++d) {
      if (!(active & (1u << d))) continue;
      const double gn = sgn[d] * red[d];
      rnorm[d] = sqrt(gn);
      const bool mach = (rnorm[d] + 1.0 <= 1.0);
      const bool solved = (rnorm[d] <= eps[d]) || mach;
      if (!solved) {
        beta[d] = gn / gamma[d];
        pn2[d] = gn + (beta[d] * beta[d]) * pn2[d];
        gamma[d] = gn;
      }
      its[d] += 1;
      const bool tired = its[d] >= cfg.itmax;
      if (!(solved || tired)) cont |= 1u << d;
    }
    active = cont;
    first = false;
    rc ^= 1;
    pc ^= 1;
  }
#pragma unroll
  for (int d = 0; d < NS; ++d) rnorm_out[d] = rnorm[d];
  return true;
}

// ---------------------------------------------------------------- GMRES
// Krylov.jl 0.9.5 gmres! with left preconditioner M, N = I, restart = false
// (the basis grows up to itmax vectors), no reorthogonalisation: modified
// Gram-Schmidt Arnoldi, QR of the Hessenberg matrix by Givens rotations
// (SymOrtho, sym_givens), back substitution for y at the end, x = V y.
// Entry (krylov_start, as for BiCGSTAB): r[0] = M^{-1}(b - A x0), x = 0,
// partials <b,r>, <r,r>.  Phases of inner iteration k:
//   P1  V_k = src/div (stored; recomputed for neighbours), t = A V_k,
//       M^{-1} row-local part
//   ..  remaining M^{-1} phases, the last reduces h_1 = <V_1, q>
//   Mi  q -= h_{i-1} V_{i-1}, reduces h_i = <V_i, q>        (i = 2..k)
//   N   q -= h_k V_k, reduces <q, q>
// Every CTA's thread 0 then updates its copy of the rotations (c, s, z) and
// the new column; CTA 0 also stores the column of R for the back substitution.
__device__ __forceinline__ double sgn1(double a) { return a > 0.0 ? 1.0 : (a < 0.0 ? -1.0 : a); }

__device__ __forceinline__ void sym_givens(double a, double b, double &c, double &s, double &rho) {
  if (b == 0.0) {
    c = (a == 0.0) ? 1.0 : sgn1(a);
    s = 0.0;
    rho = fabs(a);
  } else if (a == 0.0) {
    c = 0.0;
    s = sgn1(b);
    rho = fabs(b);
  } else if (fabs(b) > fabs(a)) {
    const double t = a / b;
    s = sgn1(b) / sqrt(1.0 + t * t);
    c = s * t;
    rho = b / s;
  } else {
    const double t = b / a;
    c = sgn1(a) / sqrt(1.0 + t * t);
    s = c * t;
    rho = a / c;
  }
}

template <int NS, typename T>
__device__ __forceinline__ bool gmres(Ctx &C, const MatT<T> &A, const KWorkT<T> &w, const KCfg &cfg, int (&its)[NS],
                      double (&rnorm_out)[NS]) {
  const KParams &P = *C.P;
  const double BTOL = 1.8189894035458565e-12;   // eps(Float64)^(3/4) = 2^-39
  double red[2 * NS];
  final_sum<2 * NS>(C.part_r(), P.ntiles, C.sm, C.sm_out, red);
  const int G1 = w.gmax + 1;
  const int kmax = min(cfg.itmax, w.gmax);
  double *gws = w.gws + (size_t)vbid() * NS * 4 * G1;
  const size_t rs = (size_t)w.gmax * (w.gmax + 1) / 2;
  double beta0[NS], rnorm[NS], eps[NS], hbis[NS];
  unsigned active = 0;
#pragma unroll
  for (int d = 0; d < NS; ++d) {
    its[d] = 0;
    beta0[d] = sqrt(red[2 * d + 1]);
    rnorm[d] = beta0[d];
    hbis[d] = beta0[d];
    eps[d] = 0.0;
    if (beta0[d] == 0.0) continue;        // x = 0 is a zero-residual solution
    eps[d] = cfg.atol + cfg.rtol * rnorm[d];
    const bool solved = rnorm[d] <= eps[d], tired = 0 >= cfg.itmax;
    if (!(solved || tired)) active |= 1u << d;
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int d = 0; d < NS; ++d) gws[(size_t)d * 4 * G1 + 2 * G1] = beta0[d];   // z_1 = beta
  const unsigned ran = active;
  const T *r0 = w.r[0];
  T *qb[2] = {w.v[0], w.v[1]};
  const size_t nv = (size_t)P.n * NS;
  const int tail = precon_tail_phases(P, A, false, 1);
  int k = 0;
  while (active) {
    ++k;
    const T *src = (k == 1) ? r0 : qb[(k - 1) & 1];
    T *qn = qb[k & 1];
    T *Vk = w.V + (size_t)(k - 1) * nv;
    double div[NS];
#pragma unroll
    for (int d = 0; d < NS; ++d) div[d] = (k == 1) ? beta0[d] : hbis[d];
    auto getv = [&](int j, int d) -> T { return (T)((double)src[(size_t)j * NS + d] / div[d]); };
    // P1: V_k, t = A V_k, M^{-1} row-local part
    C.phase(PH_KRY_SPMV);
    tile_phase<NS>(C, tail == 0, [&](int i, double (&v)[NS]) {
      T y[NS], o[NS], vk[NS];
      spmv_row<NS>(A, i, getv, y);
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        vk[d] = getv(i, d);
        Vk[(size_t)i * NS + d] = vk[d];
        w.t[(size_t)i * NS + d] = y[d];
      }
      if (precon_local<NS>(P, A, i, y, o))
#pragma unroll
        for (int d = 0; d < NS; ++d) qn[(size_t)i * NS + d] = o[d];
      if (tail == 0)
#pragma unroll
        for (int d = 0; d < NS; ++d) {
          const double v1 = (k == 1) ? (double)vk[d] : (double)w.V[(size_t)i * NS + d];
          v[d] = v1 * (double)o[d];
        }
    });
    if (!C.sync()) return false;
    if (!precon_tail<NS, NS>(C, A, (const T *)w.t, qn, false, 1, [&](int i, double (&v)[NS]) {
#pragma unroll
          for (int d = 0; d < NS; ++d)
            v[d] = (double)w.V[(size_t)i * NS + d] * (double)qn[(size_t)i * NS + d];
        }))
      return false;
    double h[NS];
    final_sum<NS>(C.part_r(), P.ntiles, C.sm, C.sm_out, h);
    if (threadIdx.x == 0)
#pragma unroll
      for (int d = 0; d < NS; ++d) gws[(size_t)d * 4 * G1 + 3 * G1] = h[d];
    // modified Gram-Schmidt against V_2..V_k, each dot after the previous update
    for (int m = 2; m <= k + 1; ++m) {
      const T *Vp = w.V + (size_t)(m - 2) * nv;
      const T *Vm = w.V + (size_t)(m - 1) * nv;
      const bool norm = (m == k + 1);
      C.phase(PH_KRY_VEC);
      tile_phase<NS>(C, true, [&](int i, double (&v)[NS]) {
#pragma unroll
        for (int d = 0; d < NS; ++d) {
          const size_t q = (size_t)i * NS + d;
          const T qv = vaxpy<T>(qn[q], -h[d], Vp[q]);
          qn[q] = qv;
          v[d] = norm ? (double)qv * (double)qv : (double)Vm[q] * (double)qv;
        }
      });
      if (!C.sync()) return false;
      final_sum<NS>(C.part_r(), P.ntiles, C.sm, C.sm_out, h);
      if (!norm && threadIdx.x == 0)
#pragma unroll
        for (int d = 0; d < NS; ++d) gws[(size_t)d * 4 * G1 + 3 * G1 + (m - 1)] = h[d];
    }
#pragma unroll
    for (int d = 0; d < NS; ++d) hbis[d] = sqrt(h[d]);
    // Givens: previous rotations on the new column, then the new rotation
    if (threadIdx.x == 0) {
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        if (!(active & (1u << d))) continue;
        double *cs = gws + (size_t)d * 4 * G1, *sn = cs + G1, *zz = sn + G1, *col = zz + G1;
        for (int i = 0; i < k - 1; ++i) {
          const double tmp = cs[i] * col[i] + sn[i] * col[i + 1];
          col[i + 1] = sn[i] * col[i] - cs[i] * col[i + 1];
          col[i] = tmp;
        }
        double c_, s_, rho;
        sym_givens(col[k - 1], hbis[d], c_, s_, rho);
        cs[k - 1] = c_;
        sn[k - 1] = s_;
        col[k - 1] = rho;
        const double zeta = s_ * zz[k - 1];
        zz[k - 1] = c_ * zz[k - 1];
        zz[k] = zeta;
        C.sm_out[d] = fabs(zeta);
        if (vbid() == 0) {
          double *Rc = w.gR + (size_t)d * rs + (size_t)(k - 1) * k / 2;
          for (int i = 0; i < k; ++i) Rc[i] = col[i];
        }
      }
    }
    __syncthreads();
    unsigned cont = 0;
#pragma unroll
    for (int d = 0; d < NS; ++d) {
      if (!(active & (1u << d))) continue;
      rnorm[d] = C.sm_out[d];
      its[d] = k;
      const bool mach = (rnorm[d] + 1.0 <= 1.0);
      const bool solved = (rnorm[d] <= eps[d]) || mach;
      const bool breakdown = hbis[d] <= BTOL;
      const bool tired = k >= kmax;
      if (!(solved || tired || breakdown)) cont |= 1u << d;
    }
    __syncthreads();
    active = cont;
  }
  if (ran) {
    // R complete (CTA 0's stores) after this barrier; y by back substitution
    C.phase(PH_KRY_VEC);
    if (!C.sync()) return false;
    if (threadIdx.x == 0) {
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        if (!(ran & (1u << d))) continue;
        const int kd = its[d];
        double *zz = gws + (size_t)d * 4 * G1 + 2 * G1, *y = zz + G1;
        const double *R = w.gR + (size_t)d * rs;
        for (int i = 0; i < kd; ++i) y[i] = zz[i];
        for (int i = kd - 1; i >= 0; --i) {
          double yi = y[i];
          for (int j = kd - 1; j >= i + 1; --j) yi = yi - R[(size_t)j * (j + 1) / 2 + i] * y[j];
          const double rii = R[(size_t)i * (i + 1) / 2 + i];
          y[i] = (fabs(rii) <= BTOL) ? 0.0 : yi / rii;
        }
      }
    }
    __syncthreads();
    tile_each(C, [&](int i) {
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        if (!(ran & (1u << d))) continue;
        const double *y = gws + (size_t)d * 4 * G1 + 3 * G1;
        const size_t q = (size_t)i * NS + d;
        double acc = (double)w.x[q];
        for (int m = 0; m < its[d]; ++m) acc = acc + y[m] * (double)w.V[(size_t)m * nv + q];
        w.x[q] = (T)acc;
      }
    });
    if (!C.sync()) return false;
  }
#pragma unroll
  for (int d = 0; d < NS; ++d) rnorm_out[d] = rnorm[d];
  return true;
}

template <int NS, typename T>
__device__ __forceinline__ bool krylov(Ctx &C, const MatT<T> &A, const KWorkT<T> &w, const double *b, const KCfg &cfg,
                       int solver, int (&its)[NS], double (&rn)[NS]) {
  if (solver == SOLVER_BICGSTAB) return bicgstab<NS, T>(C, A, w, b, cfg, its, rn);
  if (solver == SOLVER_GMRES) return gmres<NS, T>(C, A, w, cfg, its, rn);
  return cg<NS, T>(C, A, w, cfg, its, rn);
}

// -------------------------------------------------------------- assembly
// Momentum row (ux/uy[/uz] share A): _discretise! with Time, Divergence(mdotf),
// -Laplacian(nueff) and -Source(grad p) (Solvers_1_SIMPLE.jl:21-35,
// Discretise_2_generated_distretisation.jl:5-81, Discretise_1_schemes.jl:11-113),
// then apply_boundary_conditions! (Discretise_4_apply_bcs.jl:7-44 with the functors
// of Discretise_3_boundary_conditions.jl:4-209), implicit_relaxation!
// (Solve_1_api.jl:54-60) and inverse_diagonal! (Solvers_0_functions.jl:77-88).
template <int NS>
__device__ __forceinline__ void momentum_row(const KParams &P, int i, bool relax, double (&b)[NS]) {
  const Mat &A = P.AU;
  const double vol = ldro(P.vol + i);
  double acc = 0.0;
  for (int k = 0; k < P.Wf; ++k) {
    const size_t e = (size_t)k * P.np + i;
    const int f = ldro(P.f_face + e);
    if (f < 0) break;
    const double ns = (double)ldro(P.f_sign + e);
    const int pos = ldro(P.f_pos + e);
    double t2;
    const double mf = P.mdot[f];
    if (P.div == DIV_UPWIND) {
      const double ap = 1.0 * (mf * ns);
      acc += jmax(ap, 0.0);
      t2 = -jmax(-ap, 0.0);
    } else {
      const int nb = ldro(P.f_nbr + e);
      const double ax = ldro(P.fcx + f) - ldro(P.ccx + i), ay = ldro(P.fcy + f) - ldro(P.ccy + i),
                   az = ldro(P.fcz + f) - ldro(P.ccz + i);
      const double bx = ldro(P.ccx + nb) - ldro(P.ccx + i), by = ldro(P.ccy + nb) - ldro(P.ccy + i),
                   bz = ldro(P.ccz + nb) - ldro(P.ccz + i);
      const double weight = sqrt((ax * ax + ay * ay) + az * az) / sqrt((bx * bx + by * by) + bz * bz);
      const double omw = 1.0 - weight;
      const double ap = 1.0 * (mf * ns);
      acc += ap * omw;
      t2 = ap * weight;
    }
    const double ap3 = -1.0 * ((-P.nueff[f]) * ldro(P.area + f)) / ldro(P.delta + f);
    acc += ap3;
    const double t3 = -ap3;
    const double base = ldro(P.f_first + e) ? 0.0 : A.val[pos];
    A.val[pos] = (base + t2) + t3;
  }
  double prev[NS];
#pragma unroll
  for (int d = 0; d < NS; ++d) { prev[d] = P.U[(size_t)i * NS + d]; b[d] = 0.0; }
  if (P.time == TIME_EULER) {
    const double rdt = 1 / P.dt;
    acc += vol * rdt;
#pragma unroll
    for (int d = 0; d < NS; ++d) b[d] += prev[d] * vol * rdt;
  }
#pragma unroll
  for (int d = 0; d < NS; ++d) b[d] += -1.0 * P.gp[(size_t)i * NS + d] * vol;
  const FieldBC &bc = P.bcU;
  for (int q = ldro(bc.a_ptr + i); q < ldro(bc.a_ptr + i + 1); ++q) {
    const int f = ldro(bc.a_face + q);
    const BcEntry &e = bc.tab[ldro(bc.a_bc + q)];
    const double ap = 1.0 * P.mdot[f];
    if (P.div == DIV_UPWIND) {
      if (e.type == BC_DIRICHLET) {
#pragma unroll
        for (int d = 0; d < NS; ++d) b[d] -= ap * e.v[d];
      } else if (e.type == BC_NEUMANN || e.type == BC_KWALL || e.type == BC_OMEGAWALL) {
        acc += jmax(ap, 0.0);
      }
    } else {
      if (e.type == BC_DIRICHLET) {
#pragma unroll
        for (int d = 0; d < NS; ++d) b[d] += 1.0 * ((-P.mdot[f]) * e.v[d]);
      } else if (e.type == BC_NEUMANN || e.type == BC_KWALL || e.type == BC_OMEGAWALL) {
        acc += ap;
      }
    }
    if (e.type == BC_DIRICHLET) {
      const double flux = P.nueff[f] * ldro(P.area + f) / ldro(P.delta + f);
      const double apl = -1.0 * (-flux);
      acc += apl;
#pragma unroll
      for (int d = 0; d < NS; ++d) b[d] += apl * e.v[d];
    }
  }
  if (relax) {
    acc /= P.aU;
#pragma unroll
    for (int d = 0; d < NS; ++d) b[d] += (1.0 - P.aU) * acc * prev[d];
  }
  A.val[ldro(A.dpos + i)] = acc;
  P.rD[i] = vol / acc;
  st<NS>(P.bU, i, b);
}

// u . S_f of a face vector field (flux!/div!: psif[fID] . (area*normal))
template <int NS>
__device__ __forceinline__ double face_dot_S(const KParams &P, const double *uf, int f) {
  const double a = ldro(P.area + f);
  double s = uf[(size_t)f * NS] * (a * ldro(P.fnx + f)) + uf[(size_t)f * NS + 1] * (a * ldro(P.fny + f));
  if (NS == 3) s = s + uf[(size_t)f * NS + 2] * (a * ldro(P.fnz + f));
  return s;
}

// Pressure row: div!(divHv, Uf) (Calculate_0_divergence.jl:75-107) then
// Laplacian(rDf, p) == Source(divHv) with BCs and setReference!
// (Solvers_1_SIMPLE.jl:37-39,154-157, Solve_1_api.jl:62-69).
template <int NS>
__device__ __forceinline__ double pressure_row(const KParams &P, int i) {
  const Mat &A = P.AP;
  const double vol = ldro(P.vol + i);
  double dv = 0.0;
  for (int k = 0; k < P.Wf; ++k) {
    const size_t e = (size_t)k * P.np + i;
    const int f = ldro(P.f_face + e);
    if (f < 0) break;
    dv += face_dot_S<NS>(P, P.UfH, f) * (double)ldro(P.f_sign + e) / vol;
  }
  for (int q = ldro(P.cb_ptr + i); q < ldro(P.cb_ptr + i + 1); ++q)
    dv += face_dot_S<NS>(P, P.UfH, ldro(P.cb_face + q)) / vol;
  P.divH[i] = dv;
  double acc = 0.0;
  for (int k = 0; k < P.Wf; ++k) {
    const size_t e = (size_t)k * P.np + i;
    const int f = ldro(P.f_face + e);
    if (f < 0) break;
    const int pos = ldro(P.f_pos + e);
    const double ap = 1.0 * ((-P.rDf[f]) * ldro(P.area + f)) / ldro(P.delta + f);
    acc += ap;
    const double base = ldro(P.f_first + e) ? 0.0 : A.val[pos];
    A.val[pos] = base + (-ap);
  }
  double b = 0.0;
  b += 1.0 * dv * vol;
  const FieldBC &bc = P.bcP;
  for (int q = ldro(bc.a_ptr + i); q < ldro(bc.a_ptr + i + 1); ++q) {
    const int f = ldro(bc.a_face + q);
    const BcEntry &e = bc.tab[ldro(bc.a_bc + q)];
    if (e.type == BC_DIRICHLET) {
      const double flux = P.rDf[f] * ldro(P.area + f) / ldro(P.delta + f);
      const double ap = 1.0 * (-flux);
      acc += ap;
      b += ap * e.v[0];
    }
  }
  if (P.has_pref && i == P.ref_cell) {
    b += acc * P.pref;
    acc += acc;
  }
  A.val[ldro(A.dpos + i)] = acc;
  P.bP[i] = b;
  return b;
}

// H! sums (Solvers_0_functions.jl:110-140): H = (b - sum_n A_cn U_n) * (1/A_cc),
// ux's matrix for every component, neighbours in face order.
template <int NS>
__device__ __forceinline__ void H_row(const KParams &P, int i, const double (&bb)[NS]) {
  const Mat &A = P.AU;
  double sum[NS];
#pragma unroll
  for (int d = 0; d < NS; ++d) sum[d] = 0.0;
  for (int k = 0; k < P.Wf; ++k) {
    const size_t e = (size_t)k * P.np + i;
    const int f = ldro(P.f_face + e);
    if (f < 0) break;
    const int nb = ldro(P.f_nbr + e);
    const double a = A.val[ldro(P.f_pos + e)];
#pragma unroll
    for (int d = 0; d < NS; ++d) sum[d] += a * P.U[(size_t)nb * NS + d];
  }
  const double rDc = 1 / A.val[ldro(A.dpos + i)];
#pragma unroll
  for (int d = 0; d < NS; ++d) P.H[(size_t)i * NS + d] = (bb[d] - sum[d]) * rDc;
}

// ------------------------------------------------------------ face fields
// interpolate! (Calculate_2_interpolation.jl:241-277) plus correct_boundaries!
// (:135-237) for a vector cell field.
template <int NS>
__device__ __forceinline__ void face_vector(const KParams &P, const double *cellv, int f, double (&u)[NS]) {
  const double w = ldro(P.wgt + f);
  const double omw = 1.0 - w;
  const int a = ldro(P.o1 + f), b = ldro(P.o2 + f);
#pragma unroll
  for (int d = 0; d < NS; ++d) u[d] = w * cellv[(size_t)a * NS + d] + omw * cellv[(size_t)b * NS + d];
  if (f < P.nbf) {
    const int bi = ldro(P.bcU.fbc + f);
    if (bi >= 0) {
      const BcEntry &e = P.bcU.tab[bi];
#pragma unroll
      for (int d = 0; d < NS; ++d) u[d] = (e.type == BC_DIRICHLET) ? e.v[d] : cellv[(size_t)a * NS + d];
    }
  }
}

// flux!(mdotf, Uf) (Solvers_0_functions.jl:65-73) from the face-interpolated U.
template <int NS>
__device__ __forceinline__ void face_mdot(const KParams &P, int f) {
  double u[NS];
  face_vector<NS>(P, P.U, f, u);
  if (P.model == 1)
#pragma unroll
    for (int d = 0; d < NS; ++d) P.UfH[(size_t)f * NS + d] = u[d];
  const double a = ldro(P.area + f);
  double m = u[0] * (a * ldro(P.fnx + f)) + u[1] * (a * ldro(P.fny + f));
  if (NS == 3) m = m + u[2] * (a * ldro(P.fnz + f));
  P.mdot[f] = m;
}

// correct_interpolation! (Calculate_0_gradient.jl:146-173), internal face f.
template <int NS>
__device__ __forceinline__ double midpoint_corrected(const KParams &P, int f) {
  const double w = 0.5;
  const int a = ldro(P.o1 + f), b = ldro(P.o2 + f);
  const double phifp = w * (P.p[a] + P.p[b]);
  const double g0 = w * (P.gp[(size_t)a * NS] + P.gp[(size_t)b * NS]);
  const double g1 = w * (P.gp[(size_t)a * NS + 1] + P.gp[(size_t)b * NS + 1]);
  const double r0 = ldro(P.fcx + f) - w * (ldro(P.ccx + a) + ldro(P.ccx + b));
  const double r1 = ldro(P.fcy + f) - w * (ldro(P.ccy + a) + ldro(P.ccy + b));
  double dt = g0 * r0 + g1 * r1;
  if (NS == 3) {
    const double g2 = w * (P.gp[(size_t)a * NS + 2] + P.gp[(size_t)b * NS + 2]);
    const double r2 = ldro(P.fcz + f) - w * (ldro(P.ccz + a) + ldro(P.ccz + b));
    dt = dt + g2 * r2;
  }
  return phifp + dt;
}

// grad!(grad p) for the scheme in use, starting from a synchronised pf of the
// first interpolation.  With correct_u the last Green-Gauss pass also applies
// correct_velocity! (Solvers_0_functions.jl:90-99): U = H - grad(p)*rD.
template <int NS>
__device__ __forceinline__ bool gradient_p(Ctx &C, bool correct_u) {
  const KParams &P = *C.P;
  const int npass = (P.grad == GRAD_MIDPOINT) ? 3 : 1;
  for (int pass = 0; pass < npass; ++pass) {
    const bool last = (pass == npass - 1);
    C.phase(PH_GRAD);
    tile_each(C, [&](int i) {
      double g[NS];
      green_gauss_row<NS>(P, P.pf, i, g);
      st<NS>(P.gp, i, g);
      if (last && correct_u) {
        const double rdi = P.rD[i];
#pragma unroll
        for (int d = 0; d < NS; ++d) P.U[(size_t)i * NS + d] = P.H[(size_t)i * NS + d] - g[d] * rdi;
      }
    });
    if (!C.sync()) return false;
    if (!last) {
      C.phase(PH_FACE);
      grid_each(P.nf - P.nbf, [&](int q) {
        const int f = P.nbf + q;
        P.pf[f] = midpoint_corrected<NS>(P, f);
      });
      if (!C.sync()) return false;
    }
  }
  return true;
}

// ------------------------------------------------------------- k-omega
// Wilcox k-omega of RANSModels_kOmega.jl:114-415 and RANSModels_functions.jl:5-88.
constexpr double KW_BPLUS = 0.09, KW_ALPHA1 = 0.52, KW_BETA1 = 0.072, KW_SIGK = 0.5, KW_SIGW = 0.5;   // get_coeffs

__device__ __forceinline__ double nut_wall_fn(double nu, double yplus, double kappa, double E) {
  return jmax(nu * (yplus * kappa / log(jmax(E * yplus, 1.0 + 1e-4)) - 1), 0.0);
}

// omega of a wall cell (constraint!/set_cell_value!, :364-448)
__device__ __forceinline__ double omega_wall(const KParams &P, const BcEntry &e, double kc, double y) {
  const double wvis = 6.0 * P.nu / (e.beta1 * (y * y));
  const double wlog = sqrt(kc) / (e.c25 * e.kappa * y);
  const double yplus = e.c25 * y * sqrt(kc) / P.nu;
  return (yplus > e.ylam) ? wlog : wvis;
}

// Transport row of k or omega: Time + Divergence(mdotf) - Laplacian(nueff) +
// Si(D) == Source(P) (:191-207) with BCs (Discretise_3_boundary_conditions.jl),
// implicit_relaxation! and, for omega, constrain_equation! (:346-399).
__device__ __forceinline__ double scalar_row(const KParams &P, const Mat &A, int i, const double *phi,
                                             const double *gam, const double *Si, const double *src,
                                             const FieldBC &bc, double alpha, int div, int time, bool omega) {
  const double vol = ldro(P.vol + i);
  double acc = 0.0;
  for (int k = 0; k < P.Wf; ++k) {
    const size_t e = (size_t)k * P.np + i;
    const int f = ldro(P.f_face + e);
    if (f < 0) break;
    const double ns = (double)ldro(P.f_sign + e);
    const int pos = ldro(P.f_pos + e);
    double t2;
    const double mf = P.mdot[f];
    if (div == DIV_UPWIND) {
      const double ap = 1.0 * (mf * ns);
      acc += jmax(ap, 0.0);
      t2 = -jmax(-ap, 0.0);
    } else {
      const int nb = ldro(P.f_nbr + e);
      const double ax = ldro(P.fcx + f) - ldro(P.ccx + i), ay = ldro(P.fcy + f) - ldro(P.ccy + i),
                   az = ldro(P.fcz + f) - ldro(P.ccz + i);
      const double bx = ldro(P.ccx + nb) - ldro(P.ccx + i), by = ldro(P.ccy + nb) - ldro(P.ccy + i),
                   bz = ldro(P.ccz + nb) - ldro(P.ccz + i);
      const double weight = sqrt((ax * ax + ay * ay) + az * az) / sqrt((bx * bx + by * by) + bz * bz);
      const double omw = 1.0 - weight;
      const double ap = 1.0 * (mf * ns);
      acc += ap * omw;
      t2 = ap * weight;
    }
    const double ap3 = -1.0 * ((-gam[f]) * ldro(P.area + f)) / ldro(P.delta + f);
    acc += ap3;
    const double t3 = -ap3;
    const double base = ldro(P.f_first + e) ? 0.0 : A.val[pos];
    A.val[pos] = (base + t2) + t3;
  }
  const double prev = phi[i];
  double b = 0.0;
  if (time == TIME_EULER) {
    const double rdt = 1 / P.dt;
    acc += vol * rdt;
    b += prev * vol * rdt;
  }
  acc += 1.0 * Si[i] * vol;
  b += 1.0 * src[i] * vol;
  for (int q = ldro(bc.a_ptr + i); q < ldro(bc.a_ptr + i + 1); ++q) {
    const int f = ldro(bc.a_face + q);
    const BcEntry &e = bc.tab[ldro(bc.a_bc + q)];
    const double ap = 1.0 * P.mdot[f];
    const bool neu = (e.type == BC_NEUMANN || e.type == BC_KWALL || e.type == BC_OMEGAWALL);
    if (div == DIV_UPWIND) {
      if (e.type == BC_DIRICHLET) b -= ap * e.v[0];
      else if (neu) acc += jmax(ap, 0.0);
    } else {
      if (e.type == BC_DIRICHLET) b += 1.0 * ((-P.mdot[f]) * e.v[0]);
      else if (neu) acc += ap;
    }
    if (e.type == BC_DIRICHLET) {
      const double flux = gam[f] * ldro(P.area + f) / ldro(P.delta + f);
      const double apl = -1.0 * (-flux);
      acc += apl;
      b += apl * e.v[0];
    }
    if (e.type == BC_OMEGAWALL) {
      const double flux = 1.0 * Si[i];
      b += flux * phi[i] * vol;
    }
  }
  acc /= alpha;
  b += (1.0 - alpha) * acc * prev;
  if (omega)
    for (int q = ldro(bc.a_ptr + i); q < ldro(bc.a_ptr + i + 1); ++q) {
      const BcEntry &e = bc.tab[ldro(bc.a_bc + q)];
      if (e.type != BC_OMEGAWALL) continue;
      const double wc = omega_wall(P, e, P.k[i], ldro(P.delta + ldro(bc.a_face + q)));
      b += acc * wc;
      acc += acc;
    }
  A.val[ldro(A.dpos + i)] = acc;
  return b;
}

// grad!(gradU, Uf, U) Orthogonal (Calculate_0_gradient.jl:106-112) for cell i:
// g[d][j] = dU_d/dx_j by Green-Gauss of the face values in UfH.
template <int NS>
__device__ __forceinline__ void grad_u_row(const KParams &P, int i, double (&g)[3][3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int j = 0; j < 3; ++j) g[d][j] = 0.0;
  for (int k = 0; k < P.Wf; ++k) {
    const size_t e = (size_t)k * P.np + i;
    const int f = ldro(P.f_face + e);
    if (f < 0) break;
    const double ns = (double)ldro(P.f_sign + e);
    const double a = ldro(P.area + f);
    const double sx = (a * ldro(P.fnx + f)) * ns, sy = (a * ldro(P.fny + f)) * ns, sz = (a * ldro(P.fnz + f)) * ns;
#pragma unroll
    for (int d = 0; d < NS; ++d) {
      const double v = P.UfH[(size_t)f * NS + d];
      g[d][0] += v * sx;
      g[d][1] += v * sy;
      if (NS == 3) g[d][2] += v * sz;
    }
  }
  const double vol = ldro(P.vol + i);
#pragma unroll
  for (int d = 0; d < NS; ++d)
#pragma unroll
    for (int j = 0; j < NS; ++j) g[d][j] /= vol;
  for (int q = ldro(P.cb_ptr + i); q < ldro(P.cb_ptr + i + 1); ++q) {
    const int f = ldro(P.cb_face + q);
    const double a = ldro(P.area + f);
    const double sx = a * ldro(P.fnx + f), sy = a * ldro(P.fny + f), sz = a * ldro(P.fnz + f);
#pragma unroll
    for (int d = 0; d < NS; ++d) {
      const double v = P.UfH[(size_t)f * NS + d];
      double bx = v * sx, by = v * sy;
      bx /= vol;
      by /= vol;
      g[d][0] += bx;
      g[d][1] += by;
      if (NS == 3) {
        double bz = v * sz;
        bz /= vol;
        g[d][2] += bz;
      }
    }
  }
}

// bound!(field, eps()) for the rows of forward level l: the reference's
// sequential loop (later cells see updated values) in level order.
__device__ __forceinline__ void bound_row(const KParams &P, double *fld, int i) {
  const double EPS = 2.220446049250313e-16;
  double sum_flux = 0.0;
  int cnt = 0;
  for (int k = 0; k < P.Wf; ++k) {
    const size_t e = (size_t)k * P.np + i;
    if (ldro(P.f_face + e) < 0) break;
    sum_flux += jmax(fld[ldro(P.f_nbr + e)], EPS);
    cnt += 1;
  }
  const double average = sum_flux / (double)cnt;
  const double fi = fld[i];
  fld[i] = jmax(jmax(fi, average * (signbit(fi) ? 1.0 : 0.0)), EPS);
}

template <int NS, typename T>
__device__ __forceinline__ bool turbulence(Ctx &C) {
  const KParams &P = *C.P;
  const double nu = P.nu;
  // production, destruction, effective diffusivities (turbulence!, :256-272)
  C.phase(PH_TURB);
  tile_each(C, [&](int i) {
    double g[3][3];
    grad_u_row<NS>(P, i, g);
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int j = 0; j < 3; ++j) P.G[(size_t)i * 9 + 3 * d + j] = g[d][j];
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < NS; ++j)
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        const double Sjk = 0.5 * (g[k][j] + g[j][k]);
        s += Sjk * Sjk;
      }
    const double pk = s * 2.0;
    P.Pw[i] = KW_ALPHA1 * pk;
    const double wi = P.w[i];
    P.Dw[i] = KW_BETA1 * wi;
    P.Dk[i] = KW_BPLUS * wi;
    double pki = P.nut[i] * pk;
    const FieldBC &bc = P.bcK;
    for (int q = ldro(bc.a_ptr + i); q < ldro(bc.a_ptr + i + 1); ++q) {   // correct_production!
      const BcEntry &e = bc.tab[ldro(bc.a_bc + q)];
      if (e.type != BC_KWALL) continue;
      const int f = ldro(bc.a_face + q);
      const double delta = ldro(P.delta + f);
      const double nx = ldro(P.fnx + f), ny = ldro(P.fny + f), nz = ldro(P.fnz + f);
      const double kc = P.k[i];
      const double uStar = e.c25 * sqrt(kc);
      const double dUdy = uStar / (e.kappa * delta);
      const double yplus = e.c25 * delta * sqrt(kc) / nu;
      const double nutw = nut_wall_fn(nu, yplus, e.kappa, e.E);
      const double ux = P.U[(size_t)i * NS] - 0.0, uy = P.U[(size_t)i * NS + 1] - 0.0;
      const double uz = (NS == 3 ? P.U[(size_t)i * NS + 2] : P.Uz2[i]) - 0.0;
      const double dn = (ux * nx + uy * ny) + uz * nz;
      const double gx = (ux - nx * dn) / delta, gy = (uy - ny * dn) / delta, gz = (uz - nz * dn) / delta;
      const double mag = sqrt((gx * gx + gy * gy) + gz * gz);
      if (yplus > e.ylam) pki = (nu + nutw) * mag * dUdy;
    }
    P.Pk[i] = pki;
  });
  grid_each(P.nf, [&](int f) {
    P.nueffw[f] = nu + KW_SIGW * P.nutf[f];
    P.nueffk[f] = nu + KW_SIGK * P.nutf[f];
  });
  if (!C.sync()) return false;
  const KWorkT<T> &wk = workP<T>(P);
  for (int eq = 0; eq < 2; ++eq) {   // omega first, then k
    const bool om = (eq == 0);
    MatT<T> A = matP<T>(P);
    A.precon = om ? P.precW : P.precK;
    double *phi = om ? P.w : P.k;
    const KCfg &cfg = om ? P.kW : P.kK;
    C.phase(PH_TURB);
    tile_each(C, [&](int i) {
      double b[1];
      b[0] = om ? scalar_row(P, P.AP, i, phi, P.nueffw, P.Dw, P.Pw, P.bcW, P.aW, P.divW, P.timeW, true)
                : scalar_row(P, P.AP, i, phi, P.nueffk, P.Dk, P.Pk, P.bcK, P.aK, P.divK, P.timeK, false);
      P.bP[i] = b[0];
      krylov_init_row<1, T>(P, P.AP, A, wk, b, phi, i, cfg.solver);
    });
    if (!C.sync()) return false;
    if (!krylov_start<1, T>(C, A, wk, P.bP, cfg.solver)) return false;
    int its[1];
    double rn[1];
    if (!krylov<1, T>(C, A, wk, P.bP, cfg, cfg.solver, its, rn)) return false;
    // run! copy-back, then constrain_boundary! for omega (:401-448)
    C.phase(PH_TURB);
    tile_each(C, [&](int i) {
      double v = (double)wk.x[i] + phi[i];
      if (om) {
        const FieldBC &bc = P.bcW;
        for (int q = ldro(bc.a_ptr + i); q < ldro(bc.a_ptr + i + 1); ++q) {
          const BcEntry &e = bc.tab[ldro(bc.a_bc + q)];
          if (e.type != BC_OMEGAWALL) continue;
          v = omega_wall(P, e, P.k[i], ldro(P.delta + ldro(bc.a_face + q)));
        }
      }
      phi[i] = v;
    });
    if (!C.sync()) return false;
    for (int l = 0; l < P.nfl; ++l) {   // bound!(phi, eps()); after k also nut = k/omega
      tile_each(C, [&](int i) {
        if (ldro(P.flev + i) != l) return;
        bound_row(P, phi, i);
        if (!om) P.nut[i] = P.k[i] / P.w[i];
      });
      if (!C.sync()) return false;
    }
  }
  // interpolate!(nutf, nut) + correct_boundaries! + correct_eddy_viscosity! (:496-536)
  // and update_nueff! (Solvers_0_functions.jl:1-11)
  C.phase(PH_TURB);
  grid_each(P.nf, [&](int f) {
    double v = face_scalar(P, P.nut, f, P.bcN, false);
    if (f < P.nbf) {
      const int bi = ldro(P.bcN.fbc + f);
      if (bi >= 0 && P.bcN.tab[bi].type == BC_NUTWALL) {
        const BcEntry &e = P.bcN.tab[bi];
        const int c = ldro(P.o1 + f);
        const double yplus = e.c25 * ldro(P.delta + f) * sqrt(P.k[c]) / nu;
        const double nutw = nut_wall_fn(nu, yplus, e.kappa, e.E);
        if (yplus > e.ylam) v = nutw;
      }
    }
    P.nutf[f] = v;
    P.nueff[f] = nu + v;
  });
  return C.sync();
}

// ------------------------------------------------------------- programs
template <int NS, typename T>
__device__ __forceinline__ void simple_program(Ctx &C, int iters, bool piso) {
  const KParams &P = *C.P;
  const bool mid = (P.grad == GRAD_MIDPOINT);
  const double nu = P.nu;
  // set-up before the loop (Solvers_1_SIMPLE.jl:114-119)
  C.phase(PH_SETUP);
  grid_each(P.nf, [&](int f) {
    face_mdot<NS>(P, f);
    P.pf[f] = face_scalar(P, P.p, f, P.bcP, mid);
    if (P.model == 1) P.nutf[f] = 0.0;   // initialise_RANS: a fresh face field
    P.nueff[f] = (P.model == 1) ? nu + 0.0 : nu;
  });
  if (!C.sync()) return;
  if (!gradient_p<NS>(C, false)) return;
  C.phase(PH_SETUP);
  int done = 0;
  for (int it = 0; it < iters; ++it) {
    done = it + 1;
    double Rit[4] = {1.0, 1.0, 1.0, 1.0};
    bool finite = true;   // Krylov residual norms of this iteration all finite
    // ---- momentum: assemble, start Krylov, set up M, solve
    const MatT<T> &AUT = matU<T>(P);
    const KWorkT<T> &wU = workU<T>(P);
    C.phase(PH_MOM_ASM);
    tile_each(C, [&](int i) {
      double b[NS];
      momentum_row<NS>(P, i, !piso, b);
      krylov_init_row<NS, T>(P, P.AU, AUT, wU, b, P.U, i, P.kU.solver);
    });
    if (!C.sync()) return;
    if (!krylov_start<NS, T>(C, AUT, wU, P.bU, P.kU.solver)) return;
    int itsU[NS];
    double rnU[NS];
    if (!krylov<NS, T>(C, AUT, wU, P.bU, P.kU, P.kU.solver, itsU, rnU)) return;
#pragma unroll
    for (int d = 0; d < NS; ++d) finite = finite && isfinite(rnU[d]);
    // run! copy-back: U = x + x0
    C.phase(PH_UPDATE);
    tile_each(C, [&](int i) {
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const size_t k = (size_t)i * NS + d;
        P.U[k] = (double)wU.x[k] + P.U[k];
      }
    });
    if (!C.sync()) return;
    // ---- residual!(R_ux..), remove_pressure_source!, H!
    C.phase(PH_RESID);
    tile_phase<2 * NS>(C, true, [&](int i, double (&v)[2 * NS]) {
      double y[NS], bb[NS];
      spmv_row<NS>(P.AU, i, [&](int j, int d) { return P.U[(size_t)j * NS + d]; }, y);
      const double vol = ldro(P.vol + i);
      ld<NS>(P.bU, i, bb);
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const double df = y[d] - bb[d];
        v[2 * d] = df * df;
        v[2 * d + 1] = bb[d] * bb[d];
        bb[d] -= -1.0 * P.gp[(size_t)i * NS + d] * vol;
      }
      st<NS>(P.bU, i, bb);
      H_row<NS>(P, i, bb);
    });
    if (!C.sync()) return;
    {
      double red[2 * NS];
      final_sum<2 * NS>(C.part_r(), P.ntiles, C.sm, C.sm_out, red);
#pragma unroll
      for (int d = 0; d < NS; ++d) Rit[d] = sqrt(red[2 * d] / (double)P.n) / sqrt(red[2 * d + 1]);
      if (vbid() == 0 && threadIdx.x == 0) {
#pragma unroll
        for (int d = 0; d < NS; ++d) {
          P.R[(size_t)it * 4 + d] = Rit[d];
          P.kry[(size_t)it * 5 + d] = itsU[d];
        }
      }
    }
    const int ncorr = piso ? 2 : 1;
    for (int corr = 0; corr < ncorr; ++corr) {
      if (corr > 0) {   // H! again with the corrected U (PISO corrector loop)
        C.phase(PH_RESID);
        tile_each(C, [&](int i) {
          double bb[NS];
          ld<NS>(P.bU, i, bb);
          H_row<NS>(P, i, bb);
        });
        if (!C.sync()) return;
      }
      // interpolate!(rDf, rD); interpolate!(Uf, Hv) + correct_boundaries!
      C.phase(PH_FACE);
      grid_each(P.nf, [&](int f) {
        const double w = ldro(P.wgt + f);
        const double omw = 1.0 - w;
        P.rDf[f] = w * P.rD[ldro(P.o1 + f)] + omw * P.rD[ldro(P.o2 + f)];
        double u[NS];
        face_vector<NS>(P, P.H, f, u);
#pragma unroll
        for (int d = 0; d < NS; ++d) P.UfH[(size_t)f * NS + d] = u[d];
      });
      if (!C.sync()) return;
      // div! + pressure assembly + Krylov start
      const MatT<T> &APT = matP<T>(P);
      const KWorkT<T> &wP = workP<T>(P);
      C.phase(PH_P_ASM);
      tile_each(C, [&](int i) {
        double b[1];
        b[0] = pressure_row<NS>(P, i);
        krylov_init_row<1, T>(P, P.AP, APT, wP, b, P.p, i, P.kP.solver);
      });
      if (!C.sync()) return;
      if (!krylov_start<1, T>(C, APT, wP, P.bP, P.kP.solver)) return;
      int itsP[1];
      double rnP[1];
      if (!krylov<1, T>(C, APT, wP, P.bP, P.kP, P.kP.solver, itsP, rnP)) return;
      finite = finite && isfinite(rnP[0]);
      // run! copy-back then explicit_relaxation!(p, prev, alpha_p)
      C.phase(PH_UPDATE);
      tile_each(C, [&](int i) {
        const double pn = (double)wP.x[i] + P.p[i];
        const double p0 = P.p[i];
        P.p[i] = p0 + P.aP * (pn - p0);
      });
      if (!C.sync()) return;
      // residual!(R_p) and the face interpolation of grad!(grad p)
      C.phase(PH_RESID);
      tile_phase<2>(C, true, [&](int i, double (&v)[2]) {
        double y[1];
        spmv_row<1>(P.AP, i, [&](int j, int d) { return P.p[j]; }, y);
        const double bb = P.bP[i];
        const double df = y[0] - bb;
        v[0] = df * df;
        v[1] = bb * bb;
      });
      grid_each(P.nf, [&](int f) { P.pf[f] = face_scalar(P, P.p, f, P.bcP, mid); });
      if (!C.sync()) return;
      {
        double red[2];
        final_sum<2>(C.part_r(), P.ntiles, C.sm, C.sm_out, red);
        Rit[3] = sqrt(red[0] / (double)P.n) / sqrt(red[1]);
        if (vbid() == 0 && threadIdx.x == 0) {
          P.R[(size_t)it * 4 + 3] = Rit[3];
          P.kry[(size_t)it * 5 + 3] = itsP[0];
        }
      }
      if (!gradient_p<NS>(C, true)) return;
      // interpolate!(Uf, U) + correct_boundaries! + flux!(mdotf, Uf)
      C.phase(PH_FACE);
      grid_each(P.nf, [&](int f) { face_mdot<NS>(P, f); });
      if (!C.sync()) return;
      if (P.model == 1 && !turbulence<NS, T>(C)) return;
    }
    // XCAL_FLAG_ABORT_ON_NAN (no reference counterpart): stop a diverged run.
    // The residuals R_* themselves may be 0/0 = NaN on a healthy run (a zero
    // right-hand side, e.g. uy at the first iteration), so the test uses the
    // Krylov residual norms, which are finite whenever A, b and x0 are.
    if (P.abort_nan) {
      if (!finite) {
        if (vbid() == 0 && threadIdx.x == 0) P.bar->nonfinite = 1;
        break;
      }
    }
    if (!piso) {
      // convergence test (Solvers_1_SIMPLE.jl:200-215); every CTA holds the
      // same residual values, so all take the same branch
      const double conv = P.conv;
      bool c = true;
#pragma unroll
      for (int d = 0; d < NS; ++d) c = c && (Rit[d] <= conv);
      c = c && (Rit[3] <= conv);
      if (c) break;
    }
  }
  if (vbid() == 0 && threadIdx.x == 0) *P.done = done;
}

__device__ __forceinline__ void solve_program(Ctx &C) {
  const KParams &P = *C.P;
  C.phase(PH_P_ASM);
  tile_each(C, [&](int i) {
    double b[1] = {P.sb[i]};
    krylov_init_row<1, double>(P, P.AU, P.AU, P.wU, b, P.U, i, P.solve_solver);
  });
  if (!C.sync()) return;
  if (!krylov_start<1, double>(C, P.AU, P.wU, P.sb, P.solve_solver)) return;
  KCfg cfg;
  cfg.solver = P.solve_solver;
  cfg.itmax = P.solve_itmax;
  cfg.atol = P.solve_atol;
  cfg.rtol = P.solve_rtol;
  int its[1];
  double rn[1];
  if (!krylov<1, double>(C, P.AU, P.wU, P.sb, cfg, P.solve_solver, its, rn)) return;
  tile_each(C, [&](int i) { P.U[i] = P.wU.x[i] + P.U[i]; });
  if (vbid() == 0 && threadIdx.x == 0) {
    P.solve_out[0] = (double)its[0];
    P.solve_out[1] = rn[0];
    *P.done = 1;
  }
}

}  // namespace

// KParams is passed by value: the fields live in the kernel's constant
// parameter bank instead of occupying registers.  T is the scalar type of
// the Krylov iterations (double: FP64 path; float: mixed path).  MB is the
// number of resident CTAs per SM the register budget is sized for: 2 (128
// registers, few spills) suits meshes with about one tile per CTA, where a
// phase is barrier-latency bound; 4 (64 registers, more spills, twice the
// warps in flight) suits large meshes, where a phase is memory-latency bound.
template <int NS, typename T, int MB>
__global__ void __launch_bounds__(TPB, MB) xcal_program_kernel(const __grid_constant__ KParams prm, int prog, int iters) {
  __shared__ double sm[8 * MAXK];
  __shared__ double sm_out[MAXK];
  __shared__ double ws[MAXTL * MAXK * 8];
  __shared__ int sm_ok;
  __shared__ unsigned long long pacc[2 * NPH];
  Ctx C;
  C.P = &prm;
  C.S.bar = prm.bar;
  C.S.mode = prm.mode;
  C.S.nb = gridDim.x;
  if (threadIdx.x == 0) {
    s_vbid = blockIdx.x;
    s_vnb = gridDim.x;
  }
  __syncthreads();
  C.S.extra = (unsigned)prm.bar_extra;
  C.S.timeout_ns = prm.bar_timeout_ns ? prm.bar_timeout_ns : BARRIER_TIMEOUT_NS;
  C.S.epoch = 0;
  C.S.ok = &sm_ok;
  C.part = prm.part;
  C.pw = 0;
  C.rev = 0;
  C.sm = sm;
  C.sm_out = sm_out;
  C.ws = ws;
  C.timers = prm.phase != nullptr && blockIdx.x == 0 && threadIdx.x == 0;
  C.tag = PH_SETUP;
  C.pacc = pacc;
  if (C.timers) {
    for (int k = 0; k < 2 * NPH; ++k) pacc[k] = 0ull;
    C.t_last = clock64();
  }
  if (prog == PROG_SOLVE) {
    if constexpr (NS == 1 && sizeof(T) == 8) solve_program(C);
  } else {
    if constexpr (NS >= 2) simple_program<NS, T>(C, iters, prog == PROG_PISO);
  }
  if (C.timers)
    for (int k = 0; k < 2 * NPH; ++k) prm.phase[k] = pacc[k];
}

// ------------------------------------------------------------- serving
// The packed serving form: one persistent launch (all of it co-resident)
// whose CTAs take cases from the host.  Each CTA polls its mail word in
// mapped host memory; the host gives a case to a group of CTAs (any CTAs,
// numbered 0..nblk-1 inside the group), which copy the case's image from
// pinned host memory into its device region, run SIMPLE to the case's
// tolerance or iteration cap with a barrier of their own, write the results
// to pinned host memory and go back to polling.  Every wait is bounded: the
// group barrier by its 2 s limit, an idle CTA by the host's heartbeat (it
// leaves when the heartbeat stops for idle_limit_ns, or on shutdown).
__device__ __forceinline__ unsigned long long ld_acquire_sys_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_sys_i32(int *p, int v) {
  asm volatile("st.release.sys.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned atom_add_acqrel_u32(unsigned *p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

template <int NS, typename T, int MB>
__global__ void __launch_bounds__(TPB, MB) xcal_serve_kernel(ServeMail *mail, const ServeCtl *ctl) {
  __shared__ double sm[8 * MAXK];
  __shared__ double sm_out[MAXK];
  __shared__ double ws[MAXTL * MAXK * 8];
  __shared__ int sm_ok;
  __shared__ unsigned long long pacc[2 * NPH];
  __shared__ ServeJob sJ;   // the job record, read once per job
  __shared__ const ServeJob *s_job;
  __shared__ int s_cmd;
  static_assert(sizeof(ServeJob) % 8 == 0, "job record copied in 8-byte words");
  ServeMail *m = mail + blockIdx.x;
  unsigned long long seen = 0;
  if (threadIdx.x == 0) seen = *(volatile unsigned long long *)&m->ack;
  for (;;) {
    if (threadIdx.x == 0) {
      int cmd = 0;
      unsigned long long hb = *(volatile const unsigned long long *)&ctl->heartbeat;
      unsigned long long t_hb = globaltimer();
      const unsigned long long limit = ctl->idle_limit_ns;
      unsigned nap = 256, polls = 0;
      for (;;) {
        const unsigned long long q = ld_acquire_sys_u64(&m->seq);
        if (q != seen) {
          seen = q;
          cmd = 1;
          break;
        }
        if ((++polls & 15u) == 0u) {
          if (*(volatile const unsigned *)&ctl->shutdown) break;
          const unsigned long long h2 = *(volatile const unsigned long long *)&ctl->heartbeat, now = globaltimer();
          if (h2 != hb) {
            hb = h2;
            t_hb = now;
          } else if (now - t_hb > limit) {
            break;
          }
        }
        __nanosleep(nap);
        if (nap < 32768u) nap <<= 1;
      }
      if (cmd) {
        // mail fields through volatile loads: the same words held earlier
        // jobs' values, which this SM may still have cached
        s_job = *(ServeJob *const volatile *)&m->job;
        s_vbid = *(volatile const int *)&m->vbid;
        s_vnb = *(volatile const int *)&m->nblk;
        *(volatile unsigned long long *)&m->ack = seen;
      }
      s_cmd = cmd;
    }
    __syncthreads();
    if (!s_cmd) return;
    // The job record and the case image live in pinned host memory whose
    // regions are reused by later jobs: read them with ld.global.cv (fetch
    // again, never from a cached line).
    {
      const unsigned long long *src = (const unsigned long long *)s_job;
      unsigned long long *dst = (unsigned long long *)&sJ;
      for (int k = threadIdx.x; k < (int)(sizeof(ServeJob) / 8); k += TPB) dst[k] = __ldcv(src + k);
    }
    __syncthreads();
    const ServeJob &J = sJ;
    const KParams &sP = sJ.prm;
    const int B = vbid(), G = vnb();
    // this CTA's share of the region: image copy, then zero part
    {
      const uint4 *src = J.src;
      uint4 *dst = J.dst;
      const unsigned long long c16 = J.copy16, z16 = J.zero16;
      for (unsigned long long q = (unsigned long long)B * TPB + threadIdx.x; q < c16; q += (unsigned long long)G * TPB)
        dst[q] = __ldcv(src + q);
      const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
      for (unsigned long long q = (unsigned long long)B * TPB + threadIdx.x; q < z16; q += (unsigned long long)G * TPB)
        dst[c16 + q] = zero;
    }
    Ctx C;
    C.P = &sP;
    C.S.bar = sP.bar;
    C.S.mode = SYNC_GRID;
    C.S.nb = G;
    C.S.extra = 0;
    C.S.timeout_ns = BARRIER_TIMEOUT_NS;
    C.S.epoch = 0;
    C.S.ok = &sm_ok;
    C.part = sP.part;
    C.pw = 0;
    C.rev = 0;
    C.sm = sm;
    C.sm_out = sm_out;
    C.ws = ws;
    C.timers = false;
    C.tag = PH_SETUP;
    C.pacc = pacc;
    C.t_last = 0;
    if (C.sync()) simple_program<NS, T>(C, J.iters, J.prog == PROG_PISO);
    C.sync();   // the run's results (fields, histories, done) complete
    // results to pinned host memory, this CTA's share
    {
      const int n = sP.n;
      const int dn = *(volatile const int *)sP.done;
      for (int q = B * TPB + threadIdx.x; q < n * NS; q += G * TPB) J.out_U[q] = sP.U[q];
      for (int q = B * TPB + threadIdx.x; q < n; q += G * TPB) J.out_p[q] = sP.p[q];
      for (int q = B * TPB + threadIdx.x; q < dn * 4; q += G * TPB) J.out_R[q] = sP.R[q];
      for (int q = B * TPB + threadIdx.x; q < dn * 5; q += G * TPB) J.out_kry[q] = sP.kry[q];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence_system();
      const unsigned prev = atom_add_acqrel_u32(J.exits, 1u);
      if (prev + 1u == (unsigned)G) {
        // last CTA of the group out: state for the host, then the group's
        // barrier word and exit count reset for the next case that uses them
        volatile Bar *b = sP.bar;
        J.out_state[0] = *(volatile const int *)sP.done;
        J.out_state[1] = b->err;
        J.out_state[2] = b->nonfinite;
        b->count = 0ull;
        b->err = 0;
        b->nonfinite = 0;
        *(volatile unsigned *)J.exits = 0u;
        __threadfence_system();
        st_release_sys_i32(J.out_state + 3, 1);
      }
    }
    __syncthreads();
  }
}

// One translation unit per instantiation (build.py compiles this file once per
// XCAL_INST value, in parallel); the launcher table lives in xcal_launch.cu.
#if defined(XCAL_INST)
#define XCAL_CAT2(a, b) a##b
#define XCAL_CAT(a, b) XCAL_CAT2(a, b)
#ifndef XCAL_MB
#define XCAL_MB 2
#endif
#if defined(XCAL_SERVE_ONLY)
template __global__ void xcal_serve_kernel<XCAL_NS, XCAL_T, XCAL_MB>(ServeMail *, const ServeCtl *);
const void *XCAL_CAT(serve_kernel_, XCAL_INST)() {
  return (const void *)xcal_serve_kernel<XCAL_NS, XCAL_T, XCAL_MB>;
}
#else
template __global__ void xcal_program_kernel<XCAL_NS, XCAL_T, XCAL_MB>(const __grid_constant__ KParams, int, int);
const void *XCAL_CAT(program_kernel_, XCAL_INST)() {
  return (const void *)xcal_program_kernel<XCAL_NS, XCAL_T, XCAL_MB>;
}
#endif
#endif

}  // namespace xcal
