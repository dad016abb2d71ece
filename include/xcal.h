/*
 * xcal.h -- C ABI of libxcal.so, the sm_100a implementation of the per-iteration
 * hot path of XCALibre's unstructured finite-volume pressure-velocity solver.
 *
 * The reference (module FVM_1D, Julia) has no FFI of its own; its operator-level
 * seam is a set of Julia functions taking Julia structs with 1-based Int64/Float64
 * vectors.  Every entry point below names the reference function it replaces
 * (paths relative to the reference project root).  A Julia `ccall` shim binds
 * these symbols one to one.
 *
 * Conventions
 *   - All indices crossing this ABI are 1-based int64 (Julia's native layout);
 *     the library converts them to 0-based int32 for the device.
 *   - Host arrays are owned by the caller; the library copies what it needs into
 *     its own device buffers and never keeps a host pointer after a call returns.
 *   - Every function returns an int status: XCAL_OK (0) or a negative XCAL_ERR_*
 *     code.  xcal_last_error() returns the message of the last failure on a
 *     context.  A context is used by one host thread at a time; each context
 *     owns one CUDA stream.
 */
#ifndef XCAL_H
#define XCAL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum {
  XCAL_PENDING = 1,          /* xcal_serve_poll: the case has not finished yet */
  XCAL_OK = 0,
  XCAL_ERR_ARG = -1,         /* invalid argument or size */
  XCAL_ERR_MESH = -2,        /* inconsistent or corrupt mesh */
  XCAL_ERR_OOM = -3,         /* device allocation failed */
  XCAL_ERR_CUDA = -4,        /* CUDA runtime error */
  XCAL_ERR_NAN = -5,         /* non-finite field values (only with XCAL_FLAG_ABORT_ON_NAN) */
  XCAL_ERR_TIMEOUT = -6,     /* a bounded device-side wait expired */
  XCAL_ERR_STATE = -7,       /* call out of order (e.g. run before case setup) */
  XCAL_ERR_IO = -8,          /* file could not be read */
  XCAL_ERR_UNSUPPORTED = -9  /* option not implemented */
};

/* ------------------------------------------------------------ enumerations */
/* boundary condition types: src/Discretise/Discretise_0_types.jl:31-78 */
enum { XCAL_BC_DIRICHLET = 0, XCAL_BC_NEUMANN = 1, XCAL_BC_KWALL = 2,
       XCAL_BC_OMEGAWALL = 3, XCAL_BC_NUTWALL = 4 };
/* schemes: src/Discretise/Discretise_0_types.jl:13-21 */
enum { XCAL_TIME_STEADY = 0, XCAL_TIME_EULER = 1 };
enum { XCAL_DIV_LINEAR = 0, XCAL_DIV_UPWIND = 1 };
enum { XCAL_LAP_LINEAR = 0 };
enum { XCAL_GRAD_ORTHOGONAL = 0, XCAL_GRAD_MIDPOINT = 1 };
/* Krylov solvers (Krylov.jl 0.9.5 CgSolver / BicgstabSolver / GmresSolver;
 * GMRES without restart, itmax <= 1000) */
enum { XCAL_SOLVER_CG = 0, XCAL_SOLVER_BICGSTAB = 1, XCAL_SOLVER_GMRES = 2 };
/* preconditioners: src/Solve/Preconditioners/preconditioners_0_types.jl:7-12 */
enum { XCAL_PRECON_DILU = 0, XCAL_PRECON_JACOBI = 1, XCAL_PRECON_NORMDIAG = 2,
       XCAL_PRECON_NONE = 3, XCAL_PRECON_ILU0 = 4 /* ILUZero.jl 0.2.0 ilu0 */ };
/* turbulence model: src/RANSModels/RANSModels_0_types.jl:10, RANSModels_kOmega.jl:127 */
enum { XCAL_MODEL_LAMINAR = 0, XCAL_MODEL_KOMEGA = 1 };
/* cell renumbering applied once at mesh upload */
enum { XCAL_RENUMBER_NONE = 0,      /* keep the caller's numbering (exact reference order) */
       XCAL_RENUMBER_RCM = 1,       /* reverse Cuthill-McKee */
       XCAL_RENUMBER_COLOR = 2 };   /* multicolour classes (2 for quad/hex meshes) */
/* arithmetic of the device path */
enum { XCAL_PREC_FP64 = 0, XCAL_PREC_MIXED = 1 };
/* fields addressable through xcal_field_set/get */
enum { XCAL_FIELD_UX = 0, XCAL_FIELD_UY = 1, XCAL_FIELD_UZ = 2, XCAL_FIELD_P = 3,
       XCAL_FIELD_K = 4, XCAL_FIELD_OMEGA = 5, XCAL_FIELD_NUT = 6 };
/* context flags */
/* XCAL_FLAG_CLUSTER: run every program as one hardware thread-block cluster
 * (at most 16 CTAs, hardware cluster barrier), the launch form that is safe
 * to overlap with other contexts' runs on the same GPU (the serving loop). */
enum { XCAL_FLAG_ABORT_ON_NAN = 1u, XCAL_FLAG_PHASE_TIMERS = 2u, XCAL_FLAG_CLUSTER = 4u };

/* ----------------------------------------------------------------- mesh */
/*
 * The reference's flattened mesh (Mesh.Mesh2 after update_mesh_format,
 * src/Mesh/Mesh_0_types.jl:34-94, src/Mesh/Mesh2D/Mesh2D_0_update_mesh.jl:5-142).
 * Faces 1..nbfaces are the boundary faces (the reference builder numbers them
 * first, src/UNV2/UNV2_3_builder.jl:97-115).  Per-cell face lists contain the
 * internal faces only, in the order of cell.faces_range.
 */
typedef struct {
  int64_t ncells, nfaces, nbfaces;
  int32_t dim;                      /* 2 = reference 2D path; 3 = hexahedral extension */
  const double *cell_centre;        /* [ncells*3] */
  const double *cell_volume;        /* [ncells]   */
  const int64_t *cell_faces_ptr;    /* [ncells+1] 1-based start of faces_range; ptr[n]=total+1 */
  const int64_t *cell_faces;        /* [total] 1-based face ids (mesh.cell_faces) */
  const int64_t *cell_neighbours;   /* [total] 1-based (mesh.cell_neighbours) */
  const int64_t *cell_nsign;        /* [total] +1/-1 (mesh.cell_nsign) */
  const int64_t *face_owner;        /* [nfaces*2] 1-based ownerCells */
  const double *face_centre;        /* [nfaces*3] */
  const double *face_normal;        /* [nfaces*3] */
  const double *face_e;             /* [nfaces*3] */
  const double *face_area;          /* [nfaces] */
  const double *face_delta;         /* [nfaces] */
  const double *face_weight;        /* [nfaces] */
  int64_t npatches;
  const int64_t *patch_ptr;         /* [npatches+1] 0-based offsets into patch_faces/cells */
  const int64_t *patch_faces;       /* 1-based boundary.facesID, concatenated */
  const int64_t *patch_cells;       /* 1-based boundary.cellsID, concatenated */
  /* Optional (nnodes = 0: absent): mesh.nodes and mesh.cell_nodes, needed
   * only by the VTK writer. */
  int64_t nnodes;
  const double *node_coords;        /* [nnodes*3] */
  const int64_t *cell_nodes_ptr;    /* [ncells+1] 1-based start of nodes_range; ptr[n]=total+1 */
  const int64_t *cell_nodes;        /* [total] 1-based node ids (mesh.cell_nodes) */
} xcal_mesh_desc;

/* ------------------------------------------------------------ case config */
/* One boundary condition: Dirichlet(:name, value) etc., patch given by its
 * 0-based index in the mesh's patch list (boundary_index, src/Mesh/Mesh_1_functions.jl:20-30).
 * Wall-function constants default to (0.41, 0.075, 0.09, 5.2, 9.8)
 * (src/Discretise/Discretise_0_types.jl:60-78). */
typedef struct {
  int32_t patch;
  int32_t type;
  double value[3];
  double kappa, beta1, cmu, B, E;
} xcal_bc;

typedef struct { int32_t time, divergence, laplacian, gradient; } xcal_schemes;   /* set_schemes */
typedef struct { int32_t solver, preconditioner, itmax, pad;
                 double convergence, relax, atol, rtol; } xcal_solver_cfg;       /* set_solver */

typedef struct {
  int32_t model;                    /* XCAL_MODEL_* */
  int32_t precision;                /* XCAL_PREC_* */
  double nu;                        /* ConstantScalar viscosity */
  xcal_schemes schemes_U, schemes_p, schemes_k, schemes_omega;
  xcal_solver_cfg solver_U, solver_p, solver_k, solver_omega;
  int32_t iterations, write_interval;   /* set_runtime */
  double dt;
  int32_t has_pref, pad0;               /* simple!(...; pref) */
  double pref;
  int32_t nbc_U, nbc_p, nbc_k, nbc_omega, nbc_nut, pad1;
  const xcal_bc *bc_U, *bc_p, *bc_k, *bc_omega, *bc_nut;  /* @assign! order */
} xcal_case;

/* ------------------------------------------------------------ entry points */
typedef struct xcal_ctx_s *xcal_ctx;

/* Context life cycle.  No reference counterpart (the reference is host-only). */
int xcal_ctx_create(int device, uint32_t flags, xcal_ctx *out);
int xcal_ctx_destroy(xcal_ctx ctx);
int xcal_last_error(xcal_ctx ctx, char *buf, size_t n);
/* SIMPLE stop tolerance: a run stops once R_ux, R_uy (R_uz) and R_p are all
 * <= tol.  The reference hard-codes 1e-7 (src/Solvers/Solvers_1_SIMPLE.jl:200-215),
 * which is the default; the serving loop uses 1e-6. */
int xcal_ctx_set_tolerance(xcal_ctx ctx, double tol);
int xcal_version(int *major, int *minor);

/* Mesh construction on the host (replaces build_mesh + update_mesh_format,
 * src/UNV2/UNV2_3_builder.jl:3-23 and src/Mesh/Mesh2D/Mesh2D_0_update_mesh.jl:5-142).
 * Builds the reference-format mesh from a UNV file; the mesh is held inside a
 * host-side handle whose arrays are read back with xcal_hmesh_counts/arrays. */
typedef struct xcal_hmesh_s *xcal_hmesh;
int xcal_hmesh_build_unv(const char *path, double scale, xcal_hmesh *out, char *err, size_t nerr);
int xcal_hmesh_counts(xcal_hmesh m, int64_t counts[8]);  /* ncells,nfaces,nbfaces,total,npatches,patchlen,nnodes,names_len */
int xcal_hmesh_desc(xcal_hmesh m, xcal_mesh_desc *desc);  /* pointers valid until free */
int xcal_hmesh_patch_names(xcal_hmesh m, char *buf, size_t n);   /* '\n'-separated */
int xcal_hmesh_free(xcal_hmesh m);
/* Host-only helpers (no device needed): wrap a caller mesh, renumber it the way
 * xcal_mesh_upload does (perm[i] = 1-based new index of cell i+1), and build
 * the device CSR pattern and DILU level sets of a host mesh. */
int xcal_hmesh_from_desc(const xcal_mesh_desc *desc, xcal_hmesh *out, char *err, size_t nerr);
int xcal_hmesh_renumber(xcal_hmesh m, int32_t renumber, xcal_hmesh *out, int64_t *perm);
int xcal_hmesh_csr(xcal_hmesh m, int64_t *nnz, int32_t *row_ptr, int32_t *col,
                   int32_t *flevel, int32_t *blevel, int32_t *nlevels);

/* Upload a mesh to the device (the reference keeps the mesh in host structs;
 * this replaces Equation(mesh), src/ModelFramework/ModelFramework_0_types.jl:90-125,
 * and the preconditioner set-up, src/Solve/Preconditioners/preconditioners_2_functions.jl:4-13). */
int xcal_mesh_upload(xcal_ctx ctx, const xcal_mesh_desc *mesh, int32_t renumber);
/* perm[i] = 1-based device index of the caller's cell i+1 */
int xcal_mesh_permutation(xcal_ctx ctx, int64_t *perm, int64_t n);
/* The mesh the device works on, in the reference layout (equal to the input for
 * XCAL_RENUMBER_NONE).  Arrays must be sized with the input mesh's counts. */
int xcal_mesh_export(xcal_ctx ctx, int64_t *cell_faces_ptr, int64_t *cell_faces,
                     int64_t *cell_neighbours, int64_t *cell_nsign, int64_t *face_owner,
                     double *cell_centre, double *cell_volume, double *face_centre,
                     double *face_normal, double *face_e, double *face_area,
                     double *face_delta, double *face_weight, int64_t *patch_faces,
                     int64_t *patch_cells);
/* Integer device structures: CSR pattern (0-based, rows in device numbering)
 * and DILU forward/backward level of every row. */
int xcal_mesh_csr(xcal_ctx ctx, int64_t *nnz, int32_t *row_ptr, int32_t *col,
                  int32_t *flevel, int32_t *blevel, int32_t *nlevels);

/* Model and configuration (RANS{...}, @assign!, set_schemes, set_solver,
 * set_runtime, Configuration: src/RANSModels/RANSModels_0_types.jl:22-31,
 * src/Discretise/Discretise_0_types.jl:80-181, src/Solve/Solve_1_api.jl:5-30,
 * src/Simulate/Simulate_0_types.jl:3-8). */
int xcal_case_setup(xcal_ctx ctx, const xcal_case *cfg);

/* Field values in the caller's numbering (initialise!, src/Fields/Fields_0_types.jl:205-222). */
int xcal_field_set(xcal_ctx ctx, int32_t field, const double *host, int64_t n);
int xcal_field_get(xcal_ctx ctx, int32_t field, double *host, int64_t n);

/* simple!(model, config; pref) -> (R_ux, R_uy, R_p): src/Solvers/Solvers_1_SIMPLE.jl:3-231.
 * Runs `iterations` SIMPLE iterations (one persistent device kernel), writes the
 * residual histories (entries after convergence stay 1.0 as in the reference),
 * and optionally the Krylov iteration count of every solve (krylov_iters has
 * 5*iterations entries: ux, uy, uz, p, spare; may be NULL).  *done receives the
 * number of iterations executed (fewer when all residuals fall below 1e-7).
 * R_uz may be NULL for 2D meshes. */
int xcal_simple_run(xcal_ctx ctx, int32_t iterations, double *R_ux, double *R_uy,
                    double *R_uz, double *R_p, int32_t *krylov_iters, int32_t *done);
/* piso!(model, config; pref): src/Solvers/Solvers_2_PISO.jl:3-238 (2 correctors). */
int xcal_piso_run(xcal_ctx ctx, int32_t iterations, double *R_ux, double *R_uy,
                  double *R_uz, double *R_p, int32_t *krylov_iters, int32_t *done);
/* Autotuner (no reference counterpart): times `iterations` SIMPLE iterations
 * of the context's case in each launch form that computes the same values
 * (program build for 2 or 4 CTAs per SM, CTA count, hardware cluster or grid
 * barrier, CG with M^-1 inside its x/r phase), keeps the fastest for the
 * context, and remembers it for later contexts whose mesh falls in the same
 * class (components, power-of-two bucket of 256-cell tiles, matrix row width,
 * precision).  The case's fields are restored afterwards, so the tuning runs
 * leave no trace in the results.  Environment overrides (XCAL_SYNC, XCAL_OCC,
 * XCAL_NBLOCKS, XCAL_CG_FUSE) take precedence over a remembered choice. */
typedef struct {
  int32_t mode;             /* 1 hardware cluster barrier, 2 grid barrier */
  int32_t ctas;             /* CTAs of the launch */
  int32_t ctas_per_sm;      /* build of the program: 2 or 4 resident CTAs per SM */
  int32_t cg_fused;         /* 1: CG applies M^-1 inside its x/r phase */
  int32_t candidates;       /* forms timed */
  int32_t pad;
  double ms_per_iteration;  /* the chosen form */
  double ms_default;        /* the form chosen without tuning */
} xcal_tune_result;
int xcal_autotune(xcal_ctx ctx, int32_t iterations, xcal_tune_result *out);

/* Device time of the last run, and per-phase device cycle counters when the
 * context was created with XCAL_FLAG_PHASE_TIMERS (zeros otherwise).  The
 * reference times the whole loop with @time (src/Solvers/Solvers_1_SIMPLE.jl:125);
 * the timers split a run by phase class: the SM cycles (of the SM running CTA
 * 0) between the end of one device-wide phase and the end of the next are
 * charged to the class of the second.  Classes, in array order: */
enum {
  XCAL_PH_SETUP = 0,      /* set-up before the loop (interpolate!, flux!, grad!) */
  XCAL_PH_MOM_ASM,        /* momentum _discretise! + BCs + relaxation + Krylov start (r0 = b - A x0) */
  XCAL_PH_P_ASM,          /* div! + pressure _discretise! + BCs + setReference! + Krylov start */
  XCAL_PH_PREC_SETUP,     /* update_preconditioner! level phases and the first M^-1 */
  XCAL_PH_KRY_SPMV,       /* Krylov phases carrying a SpMV (with the fused vector updates) */
  XCAL_PH_KRY_PREC,       /* Krylov phases carrying preconditioner sweeps */
  XCAL_PH_KRY_VEC,        /* Krylov vector/dot-only phases */
  XCAL_PH_RESID,          /* residual! (+ remove_pressure_source!, H!) */
  XCAL_PH_FACE,           /* face interpolation phases (interpolate!, correct_boundaries!, flux!) */
  XCAL_PH_GRAD,           /* Green-Gauss grad! (+ correct_velocity!) */
  XCAL_PH_UPDATE,         /* run! copy-back and explicit_relaxation! */
  XCAL_PH_TURB,           /* k-omega phases outside its Krylov solves */
  XCAL_NPHASES
};
int xcal_last_run_stats(xcal_ctx ctx, double *ms, double *phase_cycles, int32_t nphases);
/* Per-phase cycles and number of phases of each class in the last run. */
int xcal_last_run_phases(xcal_ctx ctx, int32_t nphases, double *cycles, int64_t *count);

/* Assembled linear systems of the last iteration, in device numbering, CSR order:
 * which = 0 momentum (A shared by ux/uy/uz, b per component), 1 pressure.
 * Mirrors ux_eqn.equation / p_eqn.equation (src/ModelFramework/ModelFramework_0_types.jl:83-89). */
int xcal_equation_get(xcal_ctx ctx, int32_t which, double *vals, double *b0,
                      double *b1, double *b2);

/* ------------------------------------------------------- operator level
 * A model equation built by the caller from the reference's operators and
 * sources (Time, Laplacian, Divergence, Si, Source combined with +, -, ==
 * and the -> binding to Equation(mesh):
 * src/ModelFramework/ModelFramework_0_types.jl:15-133 and
 * ModelFramework_1_operations.jl:3-58), discretised and solved on the
 * context's mesh.  All arrays are in the context's device numbering (the
 * mesh of xcal_mesh_export; the caller's own numbering with
 * XCAL_RENUMBER_NONE).  Matrix values are CSR, in the order of the pattern
 * xcal_mesh_csr returns (row_ptr/col, 0-based, columns ascending), as
 * xcal_equation_get returns them. */
enum { XCAL_TERM_TIME = 0, XCAL_TERM_LAPLACIAN = 1, XCAL_TERM_DIVERGENCE = 2, XCAL_TERM_SI = 3 };
typedef struct {
  int32_t kind;         /* XCAL_TERM_* */
  int32_t scheme;       /* Time: XCAL_TIME_*; Divergence: XCAL_DIV_*; Laplacian: XCAL_LAP_LINEAR; Si: 0 */
  double sign;          /* +1 or -1, as the operator algebra sets it */
  const double *flux;   /* face field [nfaces] (Laplacian, Divergence) or cell field [ncells] (Si); NULL for Time */
} xcal_term;
typedef struct {
  double sign;          /* +1 or -1 */
  const double *field;  /* cell field [ncells] */
} xcal_source;
/* discretise!(eqn, prev, runtime) (src/Discretise/Discretise_2_generated_distretisation.jl:5-81,
 * schemes Discretise_1_schemes.jl:11-113) followed, when nbc > 0, by
 * apply_boundary_conditions!(eqn, BCs) (Discretise_4_apply_bcs.jl:7-44, functors
 * Discretise_3_boundary_conditions.jl:4-241); terms in model order.  component
 * picks the entry of vector BC values; phi (the solved field, cells) is read by
 * the Si/OmegaWallFunction condition; prev and dt by the Euler term (may be
 * NULL / 0 otherwise).  vals [nnz] and b [ncells] receive A and b. */
int xcal_assemble(xcal_ctx ctx, const xcal_term *terms, int32_t nterms, const xcal_source *sources,
                  int32_t nsources, const xcal_bc *bcs, int32_t nbc, int32_t component, const double *phi,
                  const double *prev, double dt, double *vals, double *b);
/* y = A x (SparseArrays mul!, src/Solvers/Solvers_0_functions.jl:18) on the context's pattern. */
int xcal_spmv(xcal_ctx ctx, const double *vals, const double *x, double *y);
/* update_preconditioner! then ldiv!(y, P, r) of the DILU preconditioner
 * (src/Solve/Preconditioners/preconditioners_1_DILU.jl:230-308). */
int xcal_dilu(xcal_ctx ctx, const double *vals, const double *r, double *y);
/* grad!(grad_phi) with the Orthogonal scheme (src/Calculate/Calculate_0_gradient.jl:96-112):
 * face values by interpolate! and correct_boundaries! with the given conditions
 * (Calculate_2_interpolation.jl:6-148), then green_gauss! (Calculate_1_green_gauss.jl:2-39).
 * grad [3*ncells]: x, y, z arrays of ncells each, concatenated. */
int xcal_grad(xcal_ctx ctx, const double *phi, const xcal_bc *bcs, int32_t nbc, double *grad);

/* Standalone linear solve on a caller CSR matrix: run!(eqn, setup) with
 * Krylov.jl solve!(solver, A, b, x0; M=P, itmax, atol, rtol) and the DILU/Jacobi
 * preconditioners (src/Solve/Solve_1_api.jl:32-46,
 * src/Solve/Preconditioners/preconditioners_1_DILU.jl:5-168).
 * row_ptr/col are 0-based; columns sorted within each row; pattern symmetric.
 * x holds x0 on entry and the solution on exit. */
int xcal_linear_solve(xcal_ctx ctx, int32_t solver, int32_t precon, int64_t n,
                      const int32_t *row_ptr, const int32_t *col, const double *val,
                      const double *b, double *x, int32_t itmax, double atol,
                      double rtol, int32_t *niter, double *final_rnorm);

/* residual!(R, equation, phi): R = sqrt(mean((A*x - b)^2)) / norm(b) for a CSR
 * system (0-based, columns ascending), src/Solvers/Solvers_0_functions.jl:13-63. */
int xcal_residual(xcal_ctx ctx, int64_t n, const int32_t *row_ptr, const int32_t *col,
                  const double *val, const double *x, const double *b, double *R);

/* Allocation-free residual!: for callers that cannot allocate device memory at
 * the point of the call (a host framework that owns all device memory through
 * its own pool, or a loop that must not pay cudaMalloc's device-wide
 * synchronisation).  No counterpart in the reference.  Same result as
 * xcal_residual, but all pointers are device memory (CSR 0-based, columns
 * ascending; R receives one double) and the partial sums live in a fixed
 * 1 MiB array of the library, so n is limited to 16,777,216 rows
 * (XCAL_ERR_ARG beyond).  The arrays must hold n+1 row offsets with
 * 0 <= d_row_ptr[i] <= d_row_ptr[i+1] <= d_row_ptr[n], and d_row_ptr[n]
 * column indices and values; the kernel skips (and the call then reports
 * with XCAL_ERR_ARG) any row range or column index outside those bounds, since
 * device arrays cannot be checked on the host.  The first call on a device
 * resolves the library array's address: make it before any stream capture; a
 * device reset after it is not supported.  The call synchronises the
 * context's stream; calls that overlap on the GPU share the array and race. */
int xcal_residual_noalloc(xcal_ctx ctx, int64_t n, const int32_t *d_row_ptr, const int32_t *d_col,
                          const double *d_val, const double *d_x, const double *d_b, double *d_R);

/* ------------------------------------------------------- post-processing
 * write_vtk(name, mesh, ("label", field)...) (src/VTK/VTK_writer.jl:22-116):
 * legacy ASCII unstructured grid "<name>.vtk" with POINTS, CELLS (0-based
 * node ids), CELL_TYPES (3 nodes: 5, 4 nodes: 9, more: 7) and CELL_DATA.
 * ncomp[f] = 1 writes SCALARS (data[f] = ncells values), 3 writes VECTORS
 * (data[f] = x, y, z arrays of ncells each, concatenated).  Numbers are
 * written in shortest round-trip form.  Needs the mesh's nodes. */
int xcal_vtk_write(const char *name, const xcal_mesh_desc *mesh, int32_t nfields, const char *const *labels,
                   const int32_t *ncomp, const double *const *data);
/* model2vtk(model, name) (VTK_writer.jl:3-20): the context's U and p (and k,
 * omega, nut for k-omega) in the caller's cell order. */
int xcal_model2vtk(xcal_ctx ctx, const char *name);
/* wall_shear_stress(patch, model) (src/Postprocess/Postprocess_forces.jl:61-94
 * with surface_normal_gradient, src/Calculate/Calculate_5_surface_normal_gradient.jl:20-37):
 * per face of the patch (0-based patch index), tau = (nu + nut_c) * Up/delta,
 * Up = (U_c - Uw) - ((U_c - Uw).n) n, Uw the patch's Dirichlet U value;
 * tau and pos (face centres) are [3*count] (x,y,z per face); cap = room. */
int xcal_wall_shear_stress(xcal_ctx ctx, int32_t patch, double *tau, double *pos, int64_t cap, int64_t *count);
/* pressure_force(patch, p, rho) and viscous_force(patch, U, rho, nu, nut)
 * (Postprocess_forces.jl:5-59), with the context's fields and viscosity. */
int xcal_pressure_force(xcal_ctx ctx, int32_t patch, double rho, double F[3]);
int xcal_viscous_force(xcal_ctx ctx, int32_t patch, double rho, double F[3]);

/* ------------------------------------------------------------- serving
 * A stream of independent cases on one GPU (no reference counterpart: the
 * reference solves one case per process).  The server runs one persistent
 * launch for its lifetime; every submitted case is copied (mesh, case,
 * initial fields), admitted once its device footprint fits the server's
 * device arena (allocated once at creation, so nothing is allocated on the
 * device while cases run), laid out on the host by set-up threads, and then
 * given a group of the launch's CTAs sized by its mesh (ceil(tiles of 256
 * cells / tiles_per_cta), at most max_ctas) and run to its tolerance or
 * max_iterations in that group, beside the other cases in flight.  Cases
 * arriving while others run start as CTAs and memory free up.  Each case's
 * result is the same as its run alone through xcal_simple_run with the same
 * precision and tolerance (the device arithmetic does not depend on the CTA
 * count).  Every case of a server has the mesh dimension `dim` and runs in
 * `precision` (the case's own precision field is ignored); laminar cases only.
 * While a server exists its launch holds the GPU: other kernels of the
 * process wait until xcal_serve_destroy.  The caller's arrays are not
 * referenced after xcal_serve_submit returns. */
typedef struct xcal_server_s *xcal_server;
typedef struct {
  int32_t slots;            /* cases running at once, 1..4096 (also bounded by the launch's CTAs) */
  int32_t max_iterations;   /* per-case SIMPLE iteration cap */
  int32_t renumber;         /* XCAL_RENUMBER_* for every case */
  int32_t precision;        /* XCAL_PREC_* of every case */
  double tolerance;         /* stop when all residuals <= tolerance */
  int32_t dim;              /* mesh dimension of every case: 2 or 3 */
  int32_t tiles_per_cta;    /* CTA group sizing (0: 4) */
  int32_t max_ctas;         /* largest CTA group of one case (0: 64) */
  int32_t setup_threads;    /* host threads laying cases out (0: half the cores, 2..8) */
  double device_bytes;      /* device arena, the admission budget (0: half the free memory) */
  double host_bytes;        /* pinned host staging for images and results (0: 4 GiB) */
} xcal_serve_cfg;
typedef struct {
  int32_t status;           /* XCAL_OK or the failing call's status */
  int32_t iterations;       /* SIMPLE iterations run */
  int32_t converged;        /* 1 when the tolerance was reached */
  int32_t ncells;
  double residual[4];       /* last R_ux, R_uy, R_uz, R_p */
  double queue_ms;          /* submit -> a set-up thread took the case */
  double setup_ms;          /* host layout, waiting for arena memory included */
  double run_ms;            /* case given its CTAs -> results collected */
  double total_ms;          /* submit -> result ready */
} xcal_serve_result;
typedef struct {
  int64_t submitted, completed, failed, queued, running;
  double cell_iterations;   /* sum over finished cases of cells x iterations */
  double run_ms;            /* sum of run times */
  double device_bytes;      /* device arena size */
  double device_bytes_peak; /* most arena memory held by admitted cases at once */
  int64_t grid_ctas;        /* CTAs of the serving launch */
} xcal_serve_stats;
int xcal_serve_create(int device, const xcal_serve_cfg *cfg, xcal_server *out);
/* U0 holds ux, uy, uz (3 x ncells, the caller's cell order); p0 ncells.
 * Either may be NULL (zero initial field).  *ticket identifies the case. */
int xcal_serve_submit(xcal_server s, const xcal_mesh_desc *mesh, const xcal_case *cfg,
                      const double *U0, const double *p0, int64_t *ticket);
/* wait_ms: 0 = do not wait, < 0 = wait until done.  Returns XCAL_PENDING while
 * the case runs; once done, fills *res and (when non-NULL) U (3 x ncells) and
 * p (ncells), releases the case and returns XCAL_OK (res->status carries a
 * failed case's error: XCAL_ERR_NAN for a case stopped at a non-finite
 * Krylov residual, XCAL_ERR_OOM for a case larger than the arena,
 * XCAL_ERR_UNSUPPORTED for a case of another dimension or model). */
int xcal_serve_poll(xcal_server s, int64_t ticket, int32_t wait_ms, xcal_serve_result *res,
                    double *U, double *p);
int xcal_serve_stats_get(xcal_server s, xcal_serve_stats *st);
/* Finishes the running cases, drops the queued ones, ends the launch. */
int xcal_serve_destroy(xcal_server s);

#ifdef __cplusplus
}
#endif
#endif /* XCAL_H */
