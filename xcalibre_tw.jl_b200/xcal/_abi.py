"""ctypes mirror of include/xcal.h and the loader for libxcal.so.

The library is built in-tree (``xcalibre_tw.jl_b200/csrc`` -> ``xcalibre_tw.jl_b200/libxcal.so``).
Loading fails loudly when the shared object is missing: there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "libxcal.so")

# status codes
XCAL_OK = 0
XCAL_PENDING = 1
ERRORS = {
    -1: "XCAL_ERR_ARG", -2: "XCAL_ERR_MESH", -3: "XCAL_ERR_OOM", -4: "XCAL_ERR_CUDA",
    -5: "XCAL_ERR_NAN", -6: "XCAL_ERR_TIMEOUT", -7: "XCAL_ERR_STATE", -8: "XCAL_ERR_IO",
    -9: "XCAL_ERR_UNSUPPORTED",
}
# enumerations (values fixed by xcal.h)
BC_DIRICHLET, BC_NEUMANN, BC_KWALL, BC_OMEGAWALL, BC_NUTWALL = 0, 1, 2, 3, 4
TIME_STEADY, TIME_EULER = 0, 1
DIV_LINEAR, DIV_UPWIND = 0, 1
GRAD_ORTHOGONAL, GRAD_MIDPOINT = 0, 1
SOLVER_CG, SOLVER_BICGSTAB, SOLVER_GMRES = 0, 1, 2
PRECON_DILU, PRECON_JACOBI, PRECON_NORMDIAG, PRECON_NONE, PRECON_ILU0 = 0, 1, 2, 3, 4
MODEL_LAMINAR, MODEL_KOMEGA = 0, 1
RENUMBER_NONE, RENUMBER_RCM, RENUMBER_COLOR = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
FIELD_UX, FIELD_UY, FIELD_UZ, FIELD_P, FIELD_K, FIELD_OMEGA, FIELD_NUT = range(7)
FLAG_ABORT_ON_NAN, FLAG_PHASE_TIMERS, FLAG_CLUSTER = 1, 2, 4
# phase classes of the per-phase timers (XCAL_PH_*)
PHASES = ("setup", "momentum_assembly", "pressure_assembly", "precon_setup", "krylov_spmv",
          "krylov_precon", "krylov_vector", "residual", "face", "gradient", "update", "turbulence")

P_d = C.POINTER(C.c_double)
P_i64 = C.POINTER(C.c_int64)
P_i32 = C.POINTER(C.c_int32)


class MeshDesc(C.Structure):
    _fields_ = [
        ("ncells", C.c_int64), ("nfaces", C.c_int64), ("nbfaces", C.c_int64),
        ("dim", C.c_int32),
        ("cell_centre", P_d), ("cell_volume", P_d),
        ("cell_faces_ptr", P_i64), ("cell_faces", P_i64), ("cell_neighbours", P_i64),
        ("cell_nsign", P_i64), ("face_owner", P_i64),
        ("face_centre", P_d), ("face_normal", P_d), ("face_e", P_d),
        ("face_area", P_d), ("face_delta", P_d), ("face_weight", P_d),
        ("npatches", C.c_int64), ("patch_ptr", P_i64), ("patch_faces", P_i64),
        ("patch_cells", P_i64),
        ("nnodes", C.c_int64), ("node_coords", P_d), ("cell_nodes_ptr", P_i64), ("cell_nodes", P_i64),
    ]


class BC(C.Structure):
    _fields_ = [("patch", C.c_int32), ("type", C.c_int32), ("value", C.c_double * 3),
                ("kappa", C.c_double), ("beta1", C.c_double), ("cmu", C.c_double),
                ("B", C.c_double), ("E", C.c_double)]


class Schemes(C.Structure):
    _fields_ = [("time", C.c_int32), ("divergence", C.c_int32), ("laplacian", C.c_int32),
                ("gradient", C.c_int32)]


class SolverCfg(C.Structure):
    _fields_ = [("solver", C.c_int32), ("preconditioner", C.c_int32), ("itmax", C.c_int32),
                ("pad", C.c_int32), ("convergence", C.c_double), ("relax", C.c_double),
                ("atol", C.c_double), ("rtol", C.c_double)]


class Case(C.Structure):
    _fields_ = [
        ("model", C.c_int32), ("precision", C.c_int32), ("nu", C.c_double),
        ("schemes_U", Schemes), ("schemes_p", Schemes), ("schemes_k", Schemes),
        ("schemes_omega", Schemes),
        ("solver_U", SolverCfg), ("solver_p", SolverCfg), ("solver_k", SolverCfg),
        ("solver_omega", SolverCfg),
        ("iterations", C.c_int32), ("write_interval", C.c_int32), ("dt", C.c_double),
        ("has_pref", C.c_int32), ("pad0", C.c_int32), ("pref", C.c_double),
        ("nbc_U", C.c_int32), ("nbc_p", C.c_int32), ("nbc_k", C.c_int32),
        ("nbc_omega", C.c_int32), ("nbc_nut", C.c_int32), ("pad1", C.c_int32),
        ("bc_U", C.POINTER(BC)), ("bc_p", C.POINTER(BC)), ("bc_k", C.POINTER(BC)),
        ("bc_omega", C.POINTER(BC)), ("bc_nut", C.POINTER(BC)),
    ]


TERM_TIME, TERM_LAPLACIAN, TERM_DIVERGENCE, TERM_SI = 0, 1, 2, 3


class Term(C.Structure):
    _fields_ = [("kind", C.c_int32), ("scheme", C.c_int32), ("sign", C.c_double), ("flux", P_d)]


class Source(C.Structure):
    _fields_ = [("sign", C.c_double), ("field", P_d)]


class TuneResult(C.Structure):
    _fields_ = [("mode", C.c_int32), ("ctas", C.c_int32), ("ctas_per_sm", C.c_int32), ("cg_fused", C.c_int32),
                ("candidates", C.c_int32), ("pad", C.c_int32), ("ms_per_iteration", C.c_double),
                ("ms_default", C.c_double)]


class ServeCfg(C.Structure):
    _fields_ = [("slots", C.c_int32), ("max_iterations", C.c_int32), ("renumber", C.c_int32),
                ("precision", C.c_int32), ("tolerance", C.c_double), ("dim", C.c_int32),
                ("tiles_per_cta", C.c_int32), ("max_ctas", C.c_int32), ("setup_threads", C.c_int32),
                ("device_bytes", C.c_double), ("host_bytes", C.c_double)]


class ServeResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("converged", C.c_int32),
                ("ncells", C.c_int32), ("residual", C.c_double * 4), ("queue_ms", C.c_double),
                ("setup_ms", C.c_double), ("run_ms", C.c_double), ("total_ms", C.c_double)]


class ServeStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
                ("queued", C.c_int64), ("running", C.c_int64), ("cell_iterations", C.c_double),
                ("run_ms", C.c_double), ("device_bytes", C.c_double), ("device_bytes_peak", C.c_double),
                ("grid_ctas", C.c_int64)]


def dptr(a):
    return a.ctypes.data_as(P_d) if a is not None else None


def i64ptr(a):
    return a.ctypes.data_as(P_i64) if a is not None else None


def i32ptr(a):
    return a.ctypes.data_as(P_i32) if a is not None else None


# exported symbols and their signatures (also checked by the CPU test suite)
SIGNATURES = {
    "xcal_ctx_create": (C.c_int, [C.c_int, C.c_uint32, C.POINTER(C.c_void_p)]),
    "xcal_ctx_destroy": (C.c_int, [C.c_void_p]),
    "xcal_last_error": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "xcal_version": (C.c_int, [P_i32, P_i32]),
    "xcal_hmesh_build_unv": (C.c_int, [C.c_char_p, C.c_double, C.POINTER(C.c_void_p),
                                       C.c_char_p, C.c_size_t]),
    "xcal_hmesh_counts": (C.c_int, [C.c_void_p, P_i64]),
    "xcal_hmesh_desc": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc)]),
    "xcal_hmesh_patch_names": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "xcal_hmesh_free": (C.c_int, [C.c_void_p]),
    "xcal_hmesh_from_desc": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(C.c_void_p), C.c_char_p,
                                       C.c_size_t]),
    "xcal_hmesh_renumber": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p), P_i64]),
    "xcal_hmesh_csr": (C.c_int, [C.c_void_p, P_i64, P_i32, P_i32, P_i32, P_i32, P_i32]),
    "xcal_mesh_upload": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc), C.c_int32]),
    "xcal_mesh_permutation": (C.c_int, [C.c_void_p, P_i64, C.c_int64]),
    "xcal_mesh_export": (C.c_int, [C.c_void_p, P_i64, P_i64, P_i64, P_i64, P_i64,
                                   P_d, P_d, P_d, P_d, P_d, P_d, P_d, P_d, P_i64, P_i64]),
    "xcal_mesh_csr": (C.c_int, [C.c_void_p, P_i64, P_i32, P_i32, P_i32, P_i32, P_i32]),
    "xcal_case_setup": (C.c_int, [C.c_void_p, C.POINTER(Case)]),
    "xcal_field_set": (C.c_int, [C.c_void_p, C.c_int32, P_d, C.c_int64]),
    "xcal_field_get": (C.c_int, [C.c_void_p, C.c_int32, P_d, C.c_int64]),
    "xcal_simple_run": (C.c_int, [C.c_void_p, C.c_int32, P_d, P_d, P_d, P_d, P_i32, P_i32]),
    "xcal_piso_run": (C.c_int, [C.c_void_p, C.c_int32, P_d, P_d, P_d, P_d, P_i32, P_i32]),
    "xcal_last_run_stats": (C.c_int, [C.c_void_p, P_d, P_d, C.c_int32]),
    "xcal_last_run_phases": (C.c_int, [C.c_void_p, C.c_int32, P_d, P_i64]),
    "xcal_autotune": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(TuneResult)]),
    "xcal_equation_get": (C.c_int, [C.c_void_p, C.c_int32, P_d, P_d, P_d, P_d]),
    "xcal_linear_solve": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int64, P_i32,
                                    P_i32, P_d, P_d, P_d, C.c_int32, C.c_double, C.c_double,
                                    P_i32, P_d]),
    "xcal_residual": (C.c_int, [C.c_void_p, C.c_int64, P_i32, P_i32, P_d, P_d, P_d, P_d]),
    "xcal_assemble": (C.c_int, [C.c_void_p, C.POINTER(Term), C.c_int32, C.POINTER(Source), C.c_int32,
                                C.POINTER(BC), C.c_int32, C.c_int32, P_d, P_d, C.c_double, P_d, P_d]),
    "xcal_spmv": (C.c_int, [C.c_void_p, P_d, P_d, P_d]),
    "xcal_dilu": (C.c_int, [C.c_void_p, P_d, P_d, P_d]),
    "xcal_grad": (C.c_int, [C.c_void_p, P_d, C.POINTER(BC), C.c_int32, P_d]),
    "xcal_residual_noalloc": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p]),
    "xcal_ctx_set_tolerance": (C.c_int, [C.c_void_p, C.c_double]),
    "xcal_vtk_write": (C.c_int, [C.c_char_p, C.POINTER(MeshDesc), C.c_int32, C.POINTER(C.c_char_p), P_i32,
                                 C.POINTER(P_d)]),
    "xcal_model2vtk": (C.c_int, [C.c_void_p, C.c_char_p]),
    "xcal_wall_shear_stress": (C.c_int, [C.c_void_p, C.c_int32, P_d, P_d, C.c_int64, P_i64]),
    "xcal_pressure_force": (C.c_int, [C.c_void_p, C.c_int32, C.c_double, P_d]),
    "xcal_viscous_force": (C.c_int, [C.c_void_p, C.c_int32, C.c_double, P_d]),
    "xcal_serve_create": (C.c_int, [C.c_int, C.POINTER(ServeCfg), C.POINTER(C.c_void_p)]),
    "xcal_serve_submit": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc), C.POINTER(Case), P_d, P_d,
                                    P_i64]),
    "xcal_serve_poll": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.POINTER(ServeResult), P_d,
                                  P_d]),
    "xcal_serve_stats_get": (C.c_int, [C.c_void_p, C.POINTER(ServeStats)]),
    "xcal_serve_destroy": (C.c_int, [C.c_void_p]),
}

_lib = None


def load(path=None):
    """Load libxcal.so (built in-tree); raises if it is absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"libxcal.so not found at {p}; build it with `python __graft_entry__.py build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class XcalError(RuntimeError):
    pass


def check(status, ctx=None, what=""):
    if status == XCAL_OK:
        return
    msg = ""
    if ctx is not None:
        buf = C.create_string_buffer(1024)
        load().xcal_last_error(ctx, buf, 1024)
        msg = buf.value.decode(errors="replace")
    raise XcalError(f"{what}: {ERRORS.get(status, status)} {msg}".strip())
