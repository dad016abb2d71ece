// The persistent device program of libxcal: one launch runs `iters` SIMPLE (or
// PISO) iterations, or one standalone Krylov solve.  Phases of an iteration are
// separated by xcal::Sync barriers; see xcal_device.cuh for the arithmetic
// contract.  Reference functions are cited at each phase.
#include <cooperative_groups.h>

#include "xcal_device.cuh"
#include "xcal_kernel.h"

namespace xcal {

namespace {

enum { BC_DIRICHLET = 0, BC_NEUMANN = 1, BC_KWALL = 2, BC_OMEGAWALL = 3, BC_NUTWALL = 4 };
enum { DIV_LINEAR = 0, DIV_UPWIND = 1 };
enum { TIME_STEADY = 0, TIME_EULER = 1 };
enum { GRAD_ORTHOGONAL = 0, GRAD_MIDPOINT = 1 };
enum { SOLVER_CG = 0, SOLVER_BICGSTAB = 1 };
enum { PRECON_DILU = 0 };

struct Ctx {
  const KParams *P;
  Sync S;
  double *sm;       // [8*MAXK]
  double *sm_out;   // [MAXK]
  __device__ bool sync() { return S.sync(); }
};

// ---------------------------------------------------------------- loops
template <class F>
__device__ __forceinline__ void tile_each(const KParams &P, F f) {
  for (int tile = blockIdx.x; tile < P.ntiles; tile += gridDim.x)
#pragma unroll 1
    for (int m = 0; m < 4; ++m) {
      const int i = tile * TILE + m * TPB + threadIdx.x;
      if (i < P.n) f(i);
    }
}

template <int K, class F>
__device__ __forceinline__ void tile_reduce(Ctx &C, const int (&slot)[K], F f) {
  const KParams &P = *C.P;
  for (int tile = blockIdx.x; tile < P.ntiles; tile += gridDim.x) {
    double acc[K];
#pragma unroll 1
    for (int m = 0; m < 4; ++m) {
      const int i = tile * TILE + m * TPB + threadIdx.x;
      double v[K];
#pragma unroll
      for (int k = 0; k < K; ++k) v[k] = 0.0;
      if (i < P.n) f(i, v);
#pragma unroll
      for (int k = 0; k < K; ++k) acc[k] = (m == 0) ? v[k] : acc[k] + v[k];
    }
    block_tree<K>(acc, C.sm);
    if (threadIdx.x == 0)
#pragma unroll
      for (int k = 0; k < K; ++k) P.part[(size_t)slot[k] * P.ntiles + tile] = acc[k];
  }
}

template <class F>
__device__ __forceinline__ void grid_each(int count, F f) {
  for (int i = blockIdx.x * TPB + threadIdx.x; i < count; i += gridDim.x * TPB) f(i);
}

// ------------------------------------------------------- preconditioning
// Part of M^{-1} that needs no other row: DILU forward level 0 (and the
// backward step of rows without upper neighbours), or a diagonal scaling.
template <int NS>
__device__ __forceinline__ void precon_fused_row(const KParams &P, const Mat &A, const double (&in)[NS],
                                                 double *out, int i, unsigned amask) {
  if (A.precon == PRECON_DILU) {
    if (__ldg(P.flev + i) != 0) return;
    double o[NS];
#pragma unroll
    for (int d = 0; d < NS; ++d) o[d] = in[d];
    if (__ldg(P.blev + i) == 0) {
      const double di = A.Dinv[i];
#pragma unroll
      for (int d = 0; d < NS; ++d) o[d] = o[d] * di;
    }
#pragma unroll
    for (int d = 0; d < NS; ++d)
      if (amask & (1u << d)) out[(size_t)i * NS + d] = o[d];
  } else {
    const double di = A.Dinv[i];
#pragma unroll
    for (int d = 0; d < NS; ++d)
      if (amask & (1u << d)) out[(size_t)i * NS + d] = di * in[d];
  }
}

// Remaining levels of M^{-1} (in -> out), after a phase that ran precon_fused_row.
template <int NS>
__device__ bool precon_levels(Ctx &C, const Mat &A, const double *in, double *out, unsigned amask) {
  const KParams &P = *C.P;
  if (A.precon != PRECON_DILU) return true;
  for (int l = 1; l < P.nfl; ++l) {
    const int b = __ldg(P.fl_ptr + l), e = __ldg(P.fl_ptr + l + 1);
    grid_each(e - b, [&](int q) {
      const int i = __ldg(P.fl_rows + b + q);
      dilu_fwd_row<NS>(A, in, out, i, __ldg(P.blev + i), amask);
    });
    if (!C.sync()) return false;
  }
  for (int l = 1; l < P.nbl; ++l) {
    const int b = __ldg(P.bl_ptr + l), e = __ldg(P.bl_ptr + l + 1);
    grid_each(e - b, [&](int q) { dilu_bwd_row<NS>(A, out, __ldg(P.bl_rows + b + q), amask); });
    if (!C.sync()) return false;
  }
  return true;
}

// update_preconditioner! for levels >= 1 fused with the first application
// (level-0 rows were set up and applied in the assembly phase).
template <int NS>
__device__ bool precon_setup_apply(Ctx &C, const Mat &A, const double *in, double *out, unsigned amask) {
  const KParams &P = *C.P;
  if (A.precon != PRECON_DILU) {
    grid_each(P.n, [&](int i) {
      diag_precon_setup_row(A, i);
      const double di = A.Dinv[i];
#pragma unroll
      for (int d = 0; d < NS; ++d) out[(size_t)i * NS + d] = di * in[(size_t)i * NS + d];
    });
    return C.sync();
  }
  for (int l = 1; l < P.nfl; ++l) {
    const int b = __ldg(P.fl_ptr + l), e = __ldg(P.fl_ptr + l + 1);
    grid_each(e - b, [&](int q) {
      const int i = __ldg(P.fl_rows + b + q);
      dilu_setup_row(A, i);
      dilu_fwd_row<NS>(A, in, out, i, __ldg(P.blev + i), amask);
    });
    if (!C.sync()) return false;
  }
  for (int l = 1; l < P.nbl; ++l) {
    const int b = __ldg(P.bl_ptr + l), e = __ldg(P.bl_ptr + l + 1);
    grid_each(e - b, [&](int q) { dilu_bwd_row<NS>(A, out, __ldg(P.bl_rows + b + q), amask); });
    if (!C.sync()) return false;
  }
  return true;
}

// Krylov start for row i (Krylov.jl warm start): r0 = b - A*x0, x = 0, and the
// row-local part of the first preconditioner application.  BiCGSTAB keeps r0
// in q and preconditions into r; CG keeps r = r0 and preconditions into v.
template <int NS>
__device__ __forceinline__ void krylov_init_row(const KParams &P, const Mat &A, const KWork &w,
                                                const double (&b)[NS], const double *x0, int i,
                                                int solver) {
  double y[NS], r0[NS];
  spmv_row<NS>(A, x0, i, y);
#pragma unroll
  for (int d = 0; d < NS; ++d) {
    r0[d] = b[d] - y[d];
    w.x[(size_t)i * NS + d] = 0.0;
  }
  if (A.precon == PRECON_DILU && __ldg(P.flev + i) == 0) dilu_setup_row(A, i);
  if (solver == SOLVER_BICGSTAB) {
#pragma unroll
    for (int d = 0; d < NS; ++d) w.q[(size_t)i * NS + d] = r0[d];
    if (A.precon == PRECON_DILU) precon_fused_row<NS>(P, A, r0, w.r, i, 0xffu);
  } else {
#pragma unroll
    for (int d = 0; d < NS; ++d) w.r[(size_t)i * NS + d] = r0[d];
    if (A.precon == PRECON_DILU) precon_fused_row<NS>(P, A, r0, w.v, i, 0xffu);
  }
}

// ------------------------------------------------------------- BiCGSTAB
// Krylov.jl 0.9.5 bicgstab! with left preconditioner M, N = I, c = b.
// On entry r = M^{-1}(b - A x0), x = 0.  its[d] receives the iteration count.
template <int NS>
__device__ bool bicgstab(Ctx &C, const Mat &A, const KWork &w, const double *bb, const KCfg &cfg,
                         int (&its)[NS], double (&rnorm_out)[NS]) {
  const KParams &P = *C.P;
  double red[2 * NS];
  int slot2[2 * NS];
#pragma unroll
  for (int k = 0; k < 2 * NS; ++k) slot2[k] = k;
  int slot1[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) slot1[k] = k;
  tile_reduce<2 * NS>(C, slot2, [&](int i, double (&v)[2 * NS]) {
#pragma unroll
    for (int d = 0; d < NS; ++d) {
      const double rv = w.r[(size_t)i * NS + d];
      w.p[(size_t)i * NS + d] = rv;
      v[2 * d] = bb[(size_t)i * NS + d] * rv;
      v[2 * d + 1] = rv * rv;
    }
  });
  if (!C.sync()) return false;
  final_sum<2 * NS>(P.part, slot2, P.ntiles, C.sm, C.sm_out, red);
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
  while (active) {
#pragma unroll
    for (int d = 0; d < NS; ++d)
      if (active & (1u << d)) { its[d] += 1; rho[d] = nrho[d]; }
    // q = A y (y = p); v = M^{-1} q
    tile_each(P, [&](int i) {
      double y[NS];
      spmv_row<NS>(A, w.p, i, y);
#pragma unroll
      for (int d = 0; d < NS; ++d)
        if (active & (1u << d)) w.q[(size_t)i * NS + d] = y[d];
      precon_fused_row<NS>(P, A, y, w.v, i, active);
    });
    if (!C.sync()) return false;
    if (!precon_levels<NS>(C, A, w.q, w.v, active)) return false;
    // alpha = rho / <c, v>
    tile_reduce<NS>(C, slot1, [&](int i, double (&v)[NS]) {
#pragma unroll
      for (int d = 0; d < NS; ++d) v[d] = bb[(size_t)i * NS + d] * w.v[(size_t)i * NS + d];
    });
    if (!C.sync()) return false;
    {
      double cv[NS];
      final_sum<NS>(P.part, slot1, P.ntiles, C.sm, C.sm_out, cv);
#pragma unroll
      for (int d = 0; d < NS; ++d)
        if (active & (1u << d)) alpha[d] = rho[d] / cv[d];
    }
    // s = r - alpha*v ; x = x + alpha*y
    tile_each(P, [&](int i) {
#pragma unroll
      for (int d = 0; d < NS; ++d)
        if (active & (1u << d)) {
          const size_t k = (size_t)i * NS + d;
          w.s[k] = w.r[k] + (-alpha[d]) * w.v[k];
          w.x[k] = w.x[k] + alpha[d] * w.p[k];
        }
    });
    if (!C.sync()) return false;
    // d = A z (z = s); t = M^{-1} d
    tile_each(P, [&](int i) {
      double y[NS];
      spmv_row<NS>(A, w.s, i, y);
#pragma unroll
      for (int d = 0; d < NS; ++d)
        if (active & (1u << d)) w.q[(size_t)i * NS + d] = y[d];
      precon_fused_row<NS>(P, A, y, w.t, i, active);
    });
    if (!C.sync()) return false;
    if (!precon_levels<NS>(C, A, w.q, w.t, active)) return false;
    // omega = <t,s>/<t,t>
    tile_reduce<2 * NS>(C, slot2, [&](int i, double (&v)[2 * NS]) {
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const size_t k = (size_t)i * NS + d;
        const double tv = w.t[k];
        v[2 * d] = tv * w.s[k];
        v[2 * d + 1] = tv * tv;
      }
    });
    if (!C.sync()) return false;
    final_sum<2 * NS>(P.part, slot2, P.ntiles, C.sm, C.sm_out, red);
#pragma unroll
    for (int d = 0; d < NS; ++d)
      if (active & (1u << d)) omega[d] = red[2 * d] / red[2 * d + 1];
    // x = x + omega*z ; r = s - omega*t ; <c,r>, <r,r>
    tile_reduce<2 * NS>(C, slot2, [&](int i, double (&v)[2 * NS]) {
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const size_t k = (size_t)i * NS + d;
        double rv = w.r[k];
        if (active & (1u << d)) {
          const double sv = w.s[k];
          w.x[k] = w.x[k] + omega[d] * sv;
          rv = sv + (-omega[d]) * w.t[k];
          w.r[k] = rv;
        }
        v[2 * d] = bb[k] * rv;
        v[2 * d + 1] = rv * rv;
      }
    });
    if (!C.sync()) return false;
    final_sum<2 * NS>(P.part, slot2, P.ntiles, C.sm, C.sm_out, red);
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
    if (cont) {
      // p = p - omega*v ; p = r + beta*p
      tile_each(P, [&](int i) {
#pragma unroll
        for (int d = 0; d < NS; ++d)
          if (cont & (1u << d)) {
            const size_t k = (size_t)i * NS + d;
            double pv = w.p[k] + (-omega[d]) * w.v[k];
            w.p[k] = w.r[k] + beta[d] * pv;
          }
      });
      if (!C.sync()) return false;
    }
    active = cont;
  }
#pragma unroll
  for (int d = 0; d < NS; ++d) rnorm_out[d] = rnorm[d];
  return true;
}

// ------------------------------------------------------------------- CG
// Krylov.jl 0.9.5 cg! with preconditioner M.  The sign of <r,z> at the start
// selects the formulation: for a negative definite system CG runs on (-A)x=-b,
// i.e. <r,z> and <p,Ap> enter with their sign flipped (negation is exact).
// On entry r = b - A x0, v = M^{-1} r, x = 0.
template <int NS>
__device__ bool cg(Ctx &C, const Mat &A, const KWork &w, const KCfg &cfg, int (&its)[NS],
                   double (&rnorm_out)[NS]) {
  const KParams &P = *C.P;
  const double EPS = 2.220446049250313e-16;
  int slot1[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) slot1[k] = k;
  double red[NS];
  tile_reduce<NS>(C, slot1, [&](int i, double (&v)[NS]) {
#pragma unroll
    for (int d = 0; d < NS; ++d) {
      const size_t k = (size_t)i * NS + d;
      const double z = w.v[k];
      w.p[k] = z;
      v[d] = w.r[k] * z;
    }
  });
  if (!C.sync()) return false;
  final_sum<NS>(P.part, slot1, P.ntiles, C.sm, C.sm_out, red);
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
  while (active) {
    // Ap
    tile_each(P, [&](int i) {
      double y[NS];
      spmv_row<NS>(A, w.p, i, y);
#pragma unroll
      for (int d = 0; d < NS; ++d)
        if (active & (1u << d)) w.q[(size_t)i * NS + d] = y[d];
    });
    if (!C.sync()) return false;
    tile_reduce<NS>(C, slot1, [&](int i, double (&v)[NS]) {
#pragma unroll
      for (int d = 0; d < NS; ++d) v[d] = w.p[(size_t)i * NS + d] * w.q[(size_t)i * NS + d];
    });
    if (!C.sync()) return false;
    final_sum<NS>(P.part, slot1, P.ntiles, C.sm, C.sm_out, red);
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
    // x += alpha p ; r -= alpha Ap ; z = M^{-1} r (row-local part)
    tile_each(P, [&](int i) {
      double rr[NS];
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const size_t k = (size_t)i * NS + d;
        rr[d] = w.r[k];
        if (active & (1u << d)) {
          w.x[k] = w.x[k] + alpha[d] * w.p[k];
          rr[d] = rr[d] + (-alpha[d]) * w.q[k];
          w.r[k] = rr[d];
        }
      }
      precon_fused_row<NS>(P, A, rr, w.v, i, active);
    });
    if (!C.sync()) return false;
    if (!precon_levels<NS>(C, A, w.r, w.v, active)) return false;
    tile_reduce<NS>(C, slot1, [&](int i, double (&v)[NS]) {
#pragma unroll
      for (int d = 0; d < NS; ++d) v[d] = w.r[(size_t)i * NS + d] * w.v[(size_t)i * NS + d];
    });
    if (!C.sync()) return false;
    final_sum<NS>(P.part, slot1, P.ntiles, C.sm, C.sm_out, red);
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
    if (cont) {
      tile_each(P, [&](int i) {
#pragma unroll
        for (int d = 0; d < NS; ++d)
          if (cont & (1u << d)) {
            const size_t k = (size_t)i * NS + d;
            w.p[k] = w.v[k] + beta[d] * w.p[k];
          }
      });
      if (!C.sync()) return false;
    }
    active = cont;
  }
#pragma unroll
  for (int d = 0; d < NS; ++d) rnorm_out[d] = rnorm[d];
  return true;
}

template <int NS>
__device__ bool krylov(Ctx &C, const Mat &A, const KWork &w, const double *b, const KCfg &cfg,
                       int solver, int (&its)[NS], double (&rn)[NS]) {
  if (solver == SOLVER_BICGSTAB) return bicgstab<NS>(C, A, w, b, cfg, its, rn);
  return cg<NS>(C, A, w, cfg, its, rn);
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
  const double vol = __ldg(P.vol + i);
  double acc = 0.0;
  const int cb = __ldg(P.cf_ptr + i), ce = __ldg(P.cf_ptr + i + 1);
  for (int k = cb; k < ce; ++k) {
    const int f = __ldg(P.cf_face + k);
    const double ns = (double)__ldg(P.cf_sign + k);
    const int slot = __ldg(P.cf_slot + k);
    double t2;
    const double mf = P.mdot[f];
    if (P.div == DIV_UPWIND) {
      const double ap = 1.0 * (mf * ns);
      acc += jmax(ap, 0.0);
      t2 = -jmax(-ap, 0.0);
    } else {
      const int nb = __ldg(P.cf_nbr + k);
      const double xfx = __ldg(P.fcx + f), xfy = __ldg(P.fcy + f), xfz = __ldg(P.fcz + f);
      const double xcx = __ldg(P.ccx + i), xcy = __ldg(P.ccy + i), xcz = __ldg(P.ccz + i);
      const double xnx = __ldg(P.ccx + nb), xny = __ldg(P.ccy + nb), xnz = __ldg(P.ccz + nb);
      const double ax = xfx - xcx, ay = xfy - xcy, az = xfz - xcz;
      const double bx = xnx - xcx, by = xny - xcy, bz = xnz - xcz;
      const double weight = sqrt((ax * ax + ay * ay) + az * az) / sqrt((bx * bx + by * by) + bz * bz);
      const double omw = 1.0 - weight;
      const double ap = 1.0 * (mf * ns);
      acc += ap * omw;
      t2 = ap * weight;
    }
    const double ap3 = -1.0 * ((-P.nueff[f]) * __ldg(P.area + f)) / __ldg(P.delta + f);
    acc += ap3;
    const double t3 = -ap3;
    const double base = __ldg(P.cf_first + k) ? 0.0 : A.val[slot];
    A.val[slot] = (base + t2) + t3;
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
  for (int q = __ldg(bc.a_ptr + i); q < __ldg(bc.a_ptr + i + 1); ++q) {
    const int f = __ldg(bc.a_face + q);
    const BcEntry &e = bc.tab[__ldg(bc.a_bc + q)];
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
      const double flux = P.nueff[f] * __ldg(P.area + f) / __ldg(P.delta + f);
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
  A.val[__ldg(A.diag + i)] = acc;
  P.rD[i] = vol / acc;
#pragma unroll
  for (int d = 0; d < NS; ++d) P.bU[(size_t)i * NS + d] = b[d];
}

// Pressure row: div!(divHv, Uf) (Calculate_0_divergence.jl:75-107) then
// Laplacian(rDf, p) == Source(divHv) with BCs and setReference!
// (Solvers_1_SIMPLE.jl:37-39,154-157, Solve_1_api.jl:62-69).
template <int NS>
__device__ __forceinline__ double pressure_row(const KParams &P, int i) {
  const Mat &A = P.AP;
  const double vol = __ldg(P.vol + i);
  const int cb = __ldg(P.cf_ptr + i), ce = __ldg(P.cf_ptr + i + 1);
  double dv = 0.0;
  for (int k = cb; k < ce; ++k) {
    const int f = __ldg(P.cf_face + k);
    const double a = __ldg(P.area + f);
    double s = P.UfH[(size_t)f * NS] * (a * __ldg(P.fnx + f)) + P.UfH[(size_t)f * NS + 1] * (a * __ldg(P.fny + f));
    if (NS == 3) s = s + P.UfH[(size_t)f * NS + 2] * (a * __ldg(P.fnz + f));
    dv += s * (double)__ldg(P.cf_sign + k) / vol;
  }
  for (int q = __ldg(P.cb_ptr + i); q < __ldg(P.cb_ptr + i + 1); ++q) {
    const int f = __ldg(P.cb_face + q);
    const double a = __ldg(P.area + f);
    double s = P.UfH[(size_t)f * NS] * (a * __ldg(P.fnx + f)) + P.UfH[(size_t)f * NS + 1] * (a * __ldg(P.fny + f));
    if (NS == 3) s = s + P.UfH[(size_t)f * NS + 2] * (a * __ldg(P.fnz + f));
    dv += s / vol;
  }
  P.divH[i] = dv;
  double acc = 0.0;
  for (int k = cb; k < ce; ++k) {
    const int f = __ldg(P.cf_face + k);
    const int slot = __ldg(P.cf_slot + k);
    const double ap = 1.0 * ((-P.rDf[f]) * __ldg(P.area + f)) / __ldg(P.delta + f);
    acc += ap;
    const double base = __ldg(P.cf_first + k) ? 0.0 : A.val[slot];
    A.val[slot] = base + (-ap);
  }
  double b = 0.0;
  b += 1.0 * dv * vol;
  const FieldBC &bc = P.bcP;
  for (int q = __ldg(bc.a_ptr + i); q < __ldg(bc.a_ptr + i + 1); ++q) {
    const int f = __ldg(bc.a_face + q);
    const BcEntry &e = bc.tab[__ldg(bc.a_bc + q)];
    if (e.type == BC_DIRICHLET) {
      const double flux = P.rDf[f] * __ldg(P.area + f) / __ldg(P.delta + f);
      const double ap = 1.0 * (-flux);
      acc += ap;
      b += ap * e.v[0];
    }
  }
  if (P.has_pref && i == P.ref_cell) {
    b += acc * P.pref;
    acc += acc;
  }
  A.val[__ldg(A.diag + i)] = acc;
  P.bP[i] = b;
  return b;
}

// ------------------------------------------------------------ face fields
// interpolate! (Calculate_2_interpolation.jl:241-277) plus correct_boundaries!
// (:135-237) for a vector cell field; returns the face value in u[].
template <int NS>
__device__ __forceinline__ void face_vector(const KParams &P, const double *cellv, int f,
                                            double (&u)[NS]) {
  const double w = __ldg(P.wgt + f);
  const double omw = 1.0 - w;
  const int a = __ldg(P.o1 + f), b = __ldg(P.o2 + f);
#pragma unroll
  for (int d = 0; d < NS; ++d) u[d] = w * cellv[(size_t)a * NS + d] + omw * cellv[(size_t)b * NS + d];
  if (f < P.nbf) {
    const int bi = __ldg(P.bcU.fbc + f);
    if (bi >= 0) {
      const BcEntry &e = P.bcU.tab[bi];
#pragma unroll
      for (int d = 0; d < NS; ++d) u[d] = (e.type == BC_DIRICHLET) ? e.v[d] : cellv[(size_t)a * NS + d];
    }
  }
}

__device__ __forceinline__ double face_scalar(const KParams &P, const double *cellv, int f,
                                              const FieldBC &bc, bool midpoint) {
  const int a = __ldg(P.o1 + f), b = __ldg(P.o2 + f);
  double v;
  if (midpoint) {
    v = 0.5 * (cellv[a] + cellv[b]);
  } else {
    const double w = __ldg(P.wgt + f);
    const double omw = 1.0 - w;
    v = w * cellv[a] + omw * cellv[b];
  }
  if (f < P.nbf) {
    const int bi = __ldg(bc.fbc + f);
    if (bi >= 0) {
      const BcEntry &e = bc.tab[bi];
      v = (e.type == BC_DIRICHLET) ? e.v[0] : cellv[a];
    }
  }
  return v;
}

// flux!(mdotf, Uf) (Solvers_0_functions.jl:65-73) from the face-interpolated U.
template <int NS>
__device__ __forceinline__ void face_mdot(const KParams &P, int f) {
  double u[NS];
  face_vector<NS>(P, P.U, f, u);
  const double a = __ldg(P.area + f);
  double m = u[0] * (a * __ldg(P.fnx + f)) + u[1] * (a * __ldg(P.fny + f));
  if (NS == 3) m = m + u[2] * (a * __ldg(P.fnz + f));
  P.mdot[f] = m;
}

// green_gauss! (Calculate_1_green_gauss.jl:2-39) of the face field pf for cell i.
template <int NS>
__device__ __forceinline__ void green_gauss_row(const KParams &P, const double *pf, int i, double (&g)[NS]) {
  double r[3] = {0.0, 0.0, 0.0};
  for (int k = __ldg(P.cf_ptr + i); k < __ldg(P.cf_ptr + i + 1); ++k) {
    const int f = __ldg(P.cf_face + k);
    const double ns = (double)__ldg(P.cf_sign + k);
    const double a = __ldg(P.area + f), v = pf[f];
    r[0] += v * ((a * __ldg(P.fnx + f)) * ns);
    r[1] += v * ((a * __ldg(P.fny + f)) * ns);
    if (NS == 3) r[2] += v * ((a * __ldg(P.fnz + f)) * ns);
  }
  const double vol = __ldg(P.vol + i);
#pragma unroll
  for (int d = 0; d < NS; ++d) r[d] /= vol;
  for (int q = __ldg(P.cb_ptr + i); q < __ldg(P.cb_ptr + i + 1); ++q) {
    const int f = __ldg(P.cb_face + q);
    const double a = __ldg(P.area + f), v = pf[f];
    double bx = v * (a * __ldg(P.fnx + f)), by = v * (a * __ldg(P.fny + f));
    bx /= vol; by /= vol;
    r[0] += bx; r[1] += by;
    if (NS == 3) { double bz = v * (a * __ldg(P.fnz + f)); bz /= vol; r[2] += bz; }
  }
#pragma unroll
  for (int d = 0; d < NS; ++d) g[d] = r[d];
}

// correct_interpolation! (Calculate_0_gradient.jl:146-173), internal face f.
template <int NS>
__device__ __forceinline__ double midpoint_corrected(const KParams &P, int f) {
  const double w = 0.5;
  const int a = __ldg(P.o1 + f), b = __ldg(P.o2 + f);
  const double phifp = w * (P.p[a] + P.p[b]);
  const double g0 = w * (P.gp[(size_t)a * NS] + P.gp[(size_t)b * NS]);
  const double g1 = w * (P.gp[(size_t)a * NS + 1] + P.gp[(size_t)b * NS + 1]);
  const double r0 = __ldg(P.fcx + f) - w * (__ldg(P.ccx + a) + __ldg(P.ccx + b));
  const double r1 = __ldg(P.fcy + f) - w * (__ldg(P.ccy + a) + __ldg(P.ccy + b));
  double dt = g0 * r0 + g1 * r1;
  if (NS == 3) {
    const double g2 = w * (P.gp[(size_t)a * NS + 2] + P.gp[(size_t)b * NS + 2]);
    const double r2 = __ldg(P.fcz + f) - w * (__ldg(P.ccz + a) + __ldg(P.ccz + b));
    dt = dt + g2 * r2;
  }
  return phifp + dt;
}

// grad!(grad p) for the scheme in use, starting from a synchronised pf of the
// first interpolation.  With correct_u the last Green-Gauss pass also applies
// correct_velocity! (Solvers_0_functions.jl:90-99): U = H - grad(p)*rD.
template <int NS>
__device__ bool gradient_p(Ctx &C, bool correct_u) {
  const KParams &P = *C.P;
  const int npass = (P.grad == GRAD_MIDPOINT) ? 3 : 1;
  for (int pass = 0; pass < npass; ++pass) {
    const bool last = (pass == npass - 1);
    tile_each(P, [&](int i) {
      double g[NS];
      green_gauss_row<NS>(P, P.pf, i, g);
#pragma unroll
      for (int d = 0; d < NS; ++d) P.gp[(size_t)i * NS + d] = g[d];
      if (last && correct_u) {
        const double rdi = P.rD[i];
#pragma unroll
        for (int d = 0; d < NS; ++d) P.U[(size_t)i * NS + d] = P.H[(size_t)i * NS + d] - g[d] * rdi;
      }
    });
    if (!C.sync()) return false;
    if (!last) {
      grid_each(P.nf - P.nbf, [&](int q) {
        const int f = P.nbf + q;
        P.pf[f] = midpoint_corrected<NS>(P, f);
      });
      if (!C.sync()) return false;
    }
  }
  return true;
}

// ------------------------------------------------------------- programs
template <int NS>
__device__ void simple_program(Ctx &C, int iters, bool piso) {
  const KParams &P = *C.P;
  const bool mid = (P.grad == GRAD_MIDPOINT);
  const double nu = P.nu;
  // set-up before the loop (Solvers_1_SIMPLE.jl:114-119)
  grid_each(P.nf, [&](int f) {
    face_mdot<NS>(P, f);
    P.pf[f] = face_scalar(P, P.p, f, P.bcP, mid);
    P.nueff[f] = nu;
  });
  if (!C.sync()) return;
  if (!gradient_p<NS>(C, false)) return;
  int done = 0;
  for (int it = 0; it < iters; ++it) {
    done = it + 1;
    double Rit[4] = {1.0, 1.0, 1.0, 1.0};
    // ---- momentum: assemble, start Krylov, set up M, solve
    tile_each(P, [&](int i) {
      double b[NS];
      momentum_row<NS>(P, i, !piso, b);
      krylov_init_row<NS>(P, P.AU, P.wU, b, P.U, i, P.kU.solver);
    });
    if (!C.sync()) return;
    {
      const double *in = (P.kU.solver == SOLVER_BICGSTAB) ? P.wU.q : P.wU.r;
      double *out = (P.kU.solver == SOLVER_BICGSTAB) ? P.wU.r : P.wU.v;
      if (!precon_setup_apply<NS>(C, P.AU, in, out, 0xffu)) return;
    }
    int itsU[NS];
    double rnU[NS];
    if (!krylov<NS>(C, P.AU, P.wU, P.bU, P.kU, P.kU.solver, itsU, rnU)) return;
    tile_each(P, [&](int i) {
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const size_t k = (size_t)i * NS + d;
        P.U[k] = P.wU.x[k] + P.U[k];
      }
    });
    if (!C.sync()) return;
    // ---- residual!(R_ux..), remove_pressure_source!, H!
    {
      int slot[2 * NS];
#pragma unroll
      for (int k = 0; k < 2 * NS; ++k) slot[k] = k;
      tile_reduce<2 * NS>(C, slot, [&](int i, double (&v)[2 * NS]) {
        const Mat &A = P.AU;
        double y[NS];
        spmv_row<NS>(A, P.U, i, y);
        const double vol = __ldg(P.vol + i);
        double bb[NS], sum[NS];
#pragma unroll
        for (int d = 0; d < NS; ++d) {
          bb[d] = P.bU[(size_t)i * NS + d];
          const double df = y[d] - bb[d];
          v[2 * d] = df * df;
          v[2 * d + 1] = bb[d] * bb[d];
          bb[d] -= -1.0 * P.gp[(size_t)i * NS + d] * vol;
          P.bU[(size_t)i * NS + d] = bb[d];
          sum[d] = 0.0;
        }
        for (int k = __ldg(P.cf_ptr + i); k < __ldg(P.cf_ptr + i + 1); ++k) {
          const int nb = __ldg(P.cf_nbr + k);
          const double a = A.val[__ldg(P.cf_slot + k)];
#pragma unroll
          for (int d = 0; d < NS; ++d) sum[d] += a * P.U[(size_t)nb * NS + d];
        }
        const double Dd = A.val[__ldg(A.diag + i)];
        const double rDc = 1 / Dd;
#pragma unroll
        for (int d = 0; d < NS; ++d) P.H[(size_t)i * NS + d] = (bb[d] - sum[d]) * rDc;
      });
      if (!C.sync()) return;
      double red[2 * NS];
      final_sum<2 * NS>(P.part, slot, P.ntiles, C.sm, C.sm_out, red);
#pragma unroll
      for (int d = 0; d < NS; ++d) Rit[d] = sqrt(red[2 * d] / (double)P.n) / sqrt(red[2 * d + 1]);
      if (blockIdx.x == 0 && threadIdx.x == 0) {
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
        tile_each(P, [&](int i) {
          const Mat &A = P.AU;
          double sum[NS];
#pragma unroll
          for (int d = 0; d < NS; ++d) sum[d] = 0.0;
          for (int k = __ldg(P.cf_ptr + i); k < __ldg(P.cf_ptr + i + 1); ++k) {
            const int nb = __ldg(P.cf_nbr + k);
            const double a = A.val[__ldg(P.cf_slot + k)];
#pragma unroll
            for (int d = 0; d < NS; ++d) sum[d] += a * P.U[(size_t)nb * NS + d];
          }
          const double rDc = 1 / A.val[__ldg(A.diag + i)];
#pragma unroll
          for (int d = 0; d < NS; ++d) P.H[(size_t)i * NS + d] = (P.bU[(size_t)i * NS + d] - sum[d]) * rDc;
        });
        if (!C.sync()) return;
      }
      // interpolate!(rDf, rD); interpolate!(Uf, Hv) + correct_boundaries!
      grid_each(P.nf, [&](int f) {
        const double w = __ldg(P.wgt + f);
        const double omw = 1.0 - w;
        P.rDf[f] = w * P.rD[__ldg(P.o1 + f)] + omw * P.rD[__ldg(P.o2 + f)];
        double u[NS];
        face_vector<NS>(P, P.H, f, u);
#pragma unroll
        for (int d = 0; d < NS; ++d) P.UfH[(size_t)f * NS + d] = u[d];
      });
      if (!C.sync()) return;
      // div! + pressure assembly + Krylov start
      tile_each(P, [&](int i) {
        double b[1];
        b[0] = pressure_row<NS>(P, i);
        krylov_init_row<1>(P, P.AP, P.wP, b, P.p, i, P.kP.solver);
      });
      if (!C.sync()) return;
      {
        const double *in = (P.kP.solver == SOLVER_BICGSTAB) ? P.wP.q : P.wP.r;
        double *out = (P.kP.solver == SOLVER_BICGSTAB) ? P.wP.r : P.wP.v;
        if (!precon_setup_apply<1>(C, P.AP, in, out, 0xffu)) return;
      }
      int itsP[1];
      double rnP[1];
      if (!krylov<1>(C, P.AP, P.wP, P.bP, P.kP, P.kP.solver, itsP, rnP)) return;
      // run! copy-back then explicit_relaxation!(p, prev, alpha_p)
      tile_each(P, [&](int i) {
        const double pn = P.wP.x[i] + P.p[i];
        const double p0 = P.p[i];
        P.p[i] = p0 + P.aP * (pn - p0);
      });
      if (!C.sync()) return;
      // residual!(R_p) and the face interpolation of grad!(grad p)
      {
        int slot[2] = {0, 1};
        tile_reduce<2>(C, slot, [&](int i, double (&v)[2]) {
          double y[1];
          spmv_row<1>(P.AP, P.p, i, y);
          const double bb = P.bP[i];
          const double df = y[0] - bb;
          v[0] = df * df;
          v[1] = bb * bb;
        });
        grid_each(P.nf, [&](int f) { P.pf[f] = face_scalar(P, P.p, f, P.bcP, mid); });
        if (!C.sync()) return;
        double red[2];
        final_sum<2>(P.part, slot, P.ntiles, C.sm, C.sm_out, red);
        Rit[3] = sqrt(red[0] / (double)P.n) / sqrt(red[1]);
        if (blockIdx.x == 0 && threadIdx.x == 0) {
          P.R[(size_t)it * 4 + 3] = Rit[3];
          P.kry[(size_t)it * 5 + 3] = itsP[0];
        }
      }
      if (!gradient_p<NS>(C, true)) return;
      // interpolate!(Uf, U) + correct_boundaries! + flux!(mdotf, Uf)
      grid_each(P.nf, [&](int f) { face_mdot<NS>(P, f); });
      if (!C.sync()) return;
    }
    if (!piso) {
      // convergence test (Solvers_1_SIMPLE.jl:200-215); every CTA holds the
      // same residual values, so all take the same branch
      const double conv = 1e-7;
      bool c = true;
#pragma unroll
      for (int d = 0; d < NS; ++d) c = c && (Rit[d] <= conv);
      c = c && (Rit[3] <= conv);
      if (c) break;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *P.done = done;
}

__device__ void solve_program(Ctx &C) {
  const KParams &P = *C.P;
  tile_each(P, [&](int i) {
    double b[1] = {P.sb[i]};
    krylov_init_row<1>(P, P.AU, P.wU, b, P.U, i, P.solve_solver);
  });
  if (!C.sync()) return;
  {
    const double *in = (P.solve_solver == SOLVER_BICGSTAB) ? P.wU.q : P.wU.r;
    double *out = (P.solve_solver == SOLVER_BICGSTAB) ? P.wU.r : P.wU.v;
    if (!precon_setup_apply<1>(C, P.AU, in, out, 0xffu)) return;
  }
  KCfg cfg;
  cfg.solver = P.solve_solver; cfg.itmax = P.solve_itmax; cfg.atol = P.solve_atol; cfg.rtol = P.solve_rtol;
  int its[1];
  double rn[1];
  if (!krylov<1>(C, P.AU, P.wU, P.sb, cfg, P.solve_solver, its, rn)) return;
  tile_each(P, [&](int i) { P.U[i] = P.wU.x[i] + P.U[i]; });
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    P.solve_out[0] = (double)its[0];
    P.solve_out[1] = rn[0];
    *P.done = 1;
  }
}

}  // namespace

template <int NS>
__global__ void __launch_bounds__(TPB, 2) xcal_program_kernel(const KParams *__restrict__ pp, int prog, int iters) {
  __shared__ double sm[8 * MAXK];
  __shared__ double sm_out[MAXK];
  __shared__ int sm_ok;
  Ctx C;
  C.P = pp;
  C.S.bar = pp->bar;
  C.S.mode = pp->mode;
  C.S.nb = gridDim.x;
  C.S.epoch = 0;
  C.S.ok = &sm_ok;
  C.sm = sm;
  C.sm_out = sm_out;
  if (prog == PROG_SOLVE) {
    if (NS == 1) solve_program(C);
    return;
  }
  simple_program<NS>(C, iters, prog == PROG_PISO);
}

template __global__ void xcal_program_kernel<1>(const KParams *, int, int);
template __global__ void xcal_program_kernel<2>(const KParams *, int, int);
template __global__ void xcal_program_kernel<3>(const KParams *, int, int);

// ------------------------------------------------------------ host launch
static cudaError_t set_attrs(const void *fn, bool cluster) {
  if (cluster) return cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return cudaSuccess;
}

const void *program_kernel_ptr(int ns) {
  if (ns == 1) return (const void *)xcal_program_kernel<1>;
  if (ns == 2) return (const void *)xcal_program_kernel<2>;
  return (const void *)xcal_program_kernel<3>;
}

cudaError_t launch_program(int ns, int mode, int nblocks, const KParams *dparams, int prog, int iters,
                           cudaStream_t stream) {
  const void *fn = program_kernel_ptr(ns);
  void *args[3];
  args[0] = (void *)&dparams;
  args[1] = (void *)&prog;
  args[2] = (void *)&iters;
  if (mode == SYNC_BLOCK) {
    return cudaLaunchKernel(fn, dim3(1), dim3(TPB), args, 0, stream);
  }
  if (mode == SYNC_CLUSTER) {
    cudaError_t e = set_attrs(fn, true);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(TPB);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = nblocks;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, args);
  }
  return cudaLaunchCooperativeKernel(fn, dim3(nblocks), dim3(TPB), args, 0, stream);
}

int max_coresident_blocks(int ns, int device) {
  int per_sm = 0, sms = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, program_kernel_ptr(ns), TPB, 0);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return per_sm * sms;
}

int max_cluster_blocks(int ns) {
  const void *fn = program_kernel_ptr(ns);
  if (set_attrs(fn, true) != cudaSuccess) return 8;
  for (int c = 16; c >= 1; c >>= 1) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c);
    cfg.blockDim = dim3(TPB);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = c;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, fn, &cfg) == cudaSuccess && nclusters >= 1) return c;
  }
  return 1;
}

}  // namespace xcal
