"""Python mirror of the reference's user-facing API (module FVM_1D).

Names, argument meaning and errors follow the Julia functions they mirror:

    mesh = build_mesh(file; scale)            src/UNV2/UNV2_3_builder.jl:3-23
    mesh = update_mesh_format(mesh)           src/Mesh/Mesh2D/Mesh2D_0_update_mesh.jl:5-142
    model = RANS(Laminar, mesh=, viscosity=ConstantScalar(nu))   src/RANSModels/RANSModels_0_types.jl:22-31
    assign(model, "U", Dirichlet("inlet", [..]), ...)            @assign!, src/Discretise/Discretise_0_types.jl:80-169
    set_schemes / set_solver / set_runtime / Configuration       Discretise_0_types.jl:171-181, src/Solve/Solve_1_api.jl:5-30
    initialise(field, value)                  src/Fields/Fields_0_types.jl:205-222
    R_ux, R_uy, R_p = simple(model, config, pref=None)          src/Solvers/Solvers_1_SIMPLE.jl:3-67
    piso(model, config, pref=None)            src/Solvers/Solvers_2_PISO.jl:3-67

The whole iteration runs in libxcal.so on the GPU; this module only marshals
arguments through the C ABI of include/xcal.h.
"""
import ctypes as C
import math

import numpy as np

from . import _abi
from .mesh import Mesh2


# ------------------------------------------------------------------ fields
class ConstantScalar:
    def __init__(self, values):
        self.values = float(values)

    def __getitem__(self, i):
        return self.values


class ScalarField:
    def __init__(self, mesh, values=None):
        self.mesh = mesh
        self.values = np.zeros(mesh.ncells) if values is None else np.asarray(values, dtype=np.float64)
        self.BCs = ()


class VectorField:
    def __init__(self, mesh):
        self.mesh = mesh
        self.x = ScalarField(mesh)
        self.y = ScalarField(mesh)
        self.z = ScalarField(mesh)
        self.BCs = ()


def initialise(field, value):
    """initialise!(field, value): vectors need three components."""
    if isinstance(field, VectorField):
        v = list(value)
        if len(v) != 3:
            raise ValueError("Vectors should have 3 components")
        field.x.values[:] = float(v[0])
        field.y.values[:] = float(v[1])
        field.z.values[:] = float(v[2])
    else:
        field.values[:] = float(value)


# ------------------------------------------------------------------ schemes
class Steady: code = _abi.TIME_STEADY
class Euler: code = _abi.TIME_EULER
class Linear: code = _abi.DIV_LINEAR
class Upwind: code = _abi.DIV_UPWIND
class Orthogonal: code = _abi.GRAD_ORTHOGONAL
class Midpoint: code = _abi.GRAD_MIDPOINT


def set_schemes(time=Steady, divergence=Linear, laplacian=Linear, gradient=Orthogonal):
    if laplacian is not Linear:
        raise ValueError("only Laplacian{Linear} exists in the reference")
    return dict(time=time, divergence=divergence, laplacian=laplacian, gradient=gradient)


# --------------------------------------------------------- solvers / precon
class CgSolver: code = _abi.SOLVER_CG
class BicgstabSolver: code = _abi.SOLVER_BICGSTAB


class GmresSolver: code = _abi.SOLVER_GMRES


class DILU: code = _abi.PRECON_DILU
class Jacobi: code = _abi.PRECON_JACOBI
class NormDiagonal: code = _abi.PRECON_NORMDIAG


class ILU0: code = _abi.PRECON_ILU0


class LDL:
    code = None


def set_solver(field, solver, preconditioner, convergence, relax, itmax=100,
               atol=math.sqrt(np.finfo(np.float64).eps), rtol=1e-3):
    """set_solver(field; solver, preconditioner, convergence, relax, itmax=100,
    atol=sqrt(eps), rtol=1e-3): src/Solve/Solve_1_api.jl:5-26."""
    pc = preconditioner if isinstance(preconditioner, type) else type(preconditioner)
    return dict(solver=solver, preconditioner=pc, convergence=float(convergence),
                relax=float(relax), itmax=int(itmax), atol=float(atol), rtol=float(rtol))


def set_runtime(iterations, write_interval=-1, time_step=1.0):
    return dict(iterations=int(iterations), dt=float(time_step), write_interval=int(write_interval))


def Configuration(schemes, solvers, runtime):
    return dict(schemes=schemes, solvers=solvers, runtime=runtime)


# ------------------------------------------------------ boundary conditions
class _BC:
    type_code = None

    def __init__(self, ID, value=0.0):
        self.ID = ID.lstrip(":") if isinstance(ID, str) else ID
        self.value = value


class Dirichlet(_BC):
    type_code = _abi.BC_DIRICHLET

    def __init__(self, ID, value):
        if isinstance(value, (list, tuple, np.ndarray)) and len(value) != 3:
            raise ValueError("Only vectors with three components can be used")
        super().__init__(ID, value)


class Neumann(_BC):
    type_code = _abi.BC_NEUMANN


WALL_DEFAULTS = dict(kappa=0.41, beta1=0.075, cmu=0.09, B=5.2, E=9.8)


class KWallFunction(_BC):
    type_code = _abi.BC_KWALL

    def __init__(self, ID, value=None):
        super().__init__(ID, dict(WALL_DEFAULTS, **(value or {})))


class OmegaWallFunction(KWallFunction):
    type_code = _abi.BC_OMEGAWALL


class NutWallFunction(KWallFunction):
    type_code = _abi.BC_NUTWALL


# ------------------------------------------------------------------ models
class Laminar:
    pass


class KOmega:
    pass


class _Turb:
    def __init__(self, mesh):
        self.k = ScalarField(mesh)
        self.omega = ScalarField(mesh)
        self.nut = ScalarField(mesh)


class RANS:
    """RANS{Laminar}(mesh=, viscosity=) / RANS{KOmega}(mesh=, viscosity=)."""

    def __init__(self, kind, mesh, viscosity):
        self.kind = kind
        self.mesh = mesh
        self.nu = viscosity if isinstance(viscosity, ConstantScalar) else ConstantScalar(viscosity)
        self.U = VectorField(mesh)
        self.p = ScalarField(mesh)
        self.turbulence = _Turb(mesh) if kind is KOmega else None


def isturbulent(model):
    return model.kind is KOmega


def assign(model, field, *bcs):
    """@assign! model U (...) / @assign! model turbulence k (...).
    `field` is "U", "p", or "turbulence.k" / "k" etc."""
    name = field.split(".")[-1]
    target = getattr(model, name, None)
    if target is None and model.turbulence is not None:
        target = getattr(model.turbulence, name)
    if target is None:
        raise KeyError(f"model has no field {field!r}")
    mesh = model.mesh
    for bc in bcs:
        mesh.boundary_index(bc.ID)   # raises on unknown patch names
        if isinstance(target, VectorField):
            if isinstance(bc.value, dict):
                raise ValueError("wall functions are scalar conditions")
            if not isinstance(bc.value, (list, tuple, np.ndarray)):
                pass
            elif len(bc.value) != 3:
                raise ValueError("Vector must have 3 components")
        elif not isinstance(bc.value, (int, float, dict, np.floating)):
            raise ValueError(f"Value given to boundary {bc.ID} is not recognised")
    target.BCs = tuple(bcs)
    return model


# ---------------------------------------------------------------- mesh I/O
def build_mesh(mesh_file, scale=1.0):
    """build_mesh(file; scale): parse a UNV file and build the mesh with the
    library's host builder (same numbering rules as the reference)."""
    lib = _abi.load()
    h = C.c_void_p()
    err = C.create_string_buffer(512)
    st = lib.xcal_hmesh_build_unv(str(mesh_file).encode(), float(scale), C.byref(h), err, 512)
    if st:
        raise _abi.XcalError(f"build_mesh: {_abi.ERRORS.get(st, st)} {err.value.decode()}")
    try:
        counts = np.zeros(8, dtype=np.int64)
        lib.xcal_hmesh_counts(h, _abi.i64ptr(counts))
        d = _abi.MeshDesc()
        lib.xcal_hmesh_desc(h, C.byref(d))
        buf = C.create_string_buffer(int(counts[7]) + 16)
        lib.xcal_hmesh_patch_names(h, buf, len(buf))
        names = [s for s in buf.value.decode().split("\n") if s]
        return Mesh2.from_desc(d, names)
    finally:
        lib.xcal_hmesh_free(h)


def update_mesh_format(mesh, integer=np.int64, float=np.float64):
    """The host builder already produces the flattened layout."""
    return mesh


# ------------------------------------------------------------ case marshal
def _bc_array(field, mesh, vector):
    bcs = field.BCs
    arr = (_abi.BC * max(1, len(bcs)))()
    for i, bc in enumerate(bcs):
        e = arr[i]
        e.patch = mesh.boundary_index(bc.ID) - 1
        e.type = bc.type_code
        if isinstance(bc.value, dict):
            e.value[:] = (0.0, 0.0, 0.0)
            for k in ("kappa", "beta1", "cmu", "B", "E"):
                setattr(e, k, float(bc.value[k]))
        else:
            v = bc.value
            if isinstance(v, (list, tuple, np.ndarray)):
                e.value[:] = (float(v[0]), float(v[1]), float(v[2]))
            else:
                e.value[:] = (float(v), float(v), float(v))
            for k, dv in WALL_DEFAULTS.items():
                setattr(e, k, dv)
    return arr, len(bcs)


def _schemes(s):
    return _abi.Schemes(s["time"].code, s["divergence"].code, 0, s["gradient"].code)


def _solver(s, name):
    code = s["solver"].code
    pcode = s["preconditioner"].code
    if code is None:
        raise _abi.XcalError(f"{name}: solver {s['solver'].__name__} is not available (CG, BiCGSTAB, GMRES)")
    if pcode is None:
        raise _abi.XcalError(f"{name}: preconditioner {s['preconditioner'].__name__} is not "
                             "available (DILU, ILU0, Jacobi, NormDiagonal)")
    return _abi.SolverCfg(code, pcode, s["itmax"], 0, s["convergence"], s["relax"], s["atol"], s["rtol"])


def make_case(model, config, pref=None, precision=_abi.PREC_FP64):
    """Build the C `xcal_case` struct; returns (case, keepalive)."""
    mesh = model.mesh
    sch = config["schemes"]
    sol = config["solvers"]
    rt = config["runtime"]
    c = _abi.Case()
    c.model = _abi.MODEL_KOMEGA if isturbulent(model) else _abi.MODEL_LAMINAR
    c.precision = precision
    c.nu = model.nu.values
    c.schemes_U = _schemes(sch["U"])
    c.schemes_p = _schemes(sch["p"])
    c.solver_U = _solver(sol["U"], "U")
    c.solver_p = _solver(sol["p"], "p")
    keep = []
    bU, c.nbc_U = _bc_array(model.U, mesh, True)
    bp, c.nbc_p = _bc_array(model.p, mesh, False)
    keep += [bU, bp]
    c.bc_U = C.cast(bU, C.POINTER(_abi.BC))
    c.bc_p = C.cast(bp, C.POINTER(_abi.BC))
    if isturbulent(model):
        c.schemes_k = _schemes(sch["k"])
        c.schemes_omega = _schemes(sch["omega"])
        c.solver_k = _solver(sol["k"], "k")
        c.solver_omega = _solver(sol["omega"], "omega")
        t = model.turbulence
        bk, c.nbc_k = _bc_array(t.k, mesh, False)
        bw, c.nbc_omega = _bc_array(t.omega, mesh, False)
        bn, c.nbc_nut = _bc_array(t.nut, mesh, False)
        keep += [bk, bw, bn]
        c.bc_k = C.cast(bk, C.POINTER(_abi.BC))
        c.bc_omega = C.cast(bw, C.POINTER(_abi.BC))
        c.bc_nut = C.cast(bn, C.POINTER(_abi.BC))
    c.iterations = rt["iterations"]
    c.write_interval = rt["write_interval"]
    c.dt = rt["dt"]
    c.has_pref = 0 if pref is None else 1
    c.pref = 0.0 if pref is None else float(pref)
    return c, keep


# ----------------------------------------------------------- device solver
class Solver:
    """One device context holding a mesh, a case and the device fields."""

    def __init__(self, mesh, device=0, renumber=_abi.RENUMBER_COLOR, flags=0):
        self.lib = _abi.load()
        self.mesh = mesh
        h = C.c_void_p()
        _abi.check(self.lib.xcal_ctx_create(device, flags, C.byref(h)), None, "xcal_ctx_create")
        self.ctx = h
        _abi.check(self.lib.xcal_mesh_upload(self.ctx, C.byref(mesh.desc()), renumber), self.ctx,
                   "xcal_mesh_upload")
        self.n = mesh.ncells

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.xcal_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def setup(self, case):
        _abi.check(self.lib.xcal_case_setup(self.ctx, C.byref(case)), self.ctx, "xcal_case_setup")

    # --- post-processing (src/VTK/VTK_writer.jl, src/Postprocess/Postprocess_forces.jl)
    def model2vtk(self, name):
        """model2vtk: '<name>.vtk' with this context's U, p (k, omega, nut)."""
        _abi.check(self.lib.xcal_model2vtk(self.ctx, str(name).encode()), self.ctx, "xcal_model2vtk")

    def wall_shear_stress(self, patch):
        """wall_shear_stress(:patch, model) -> (tau [nfaces,3], face centres [nfaces,3])."""
        pid = self.mesh.boundary_index(patch) - 1
        m = int(self.mesh.patch_ptr[pid + 1] - self.mesh.patch_ptr[pid])
        tau = np.zeros(3 * m)
        pos = np.zeros(3 * m)
        cnt = np.zeros(1, dtype=np.int64)
        _abi.check(self.lib.xcal_wall_shear_stress(self.ctx, pid, _abi.dptr(tau), _abi.dptr(pos), m,
                                                   _abi.i64ptr(cnt)), self.ctx, "xcal_wall_shear_stress")
        return tau.reshape(m, 3), pos.reshape(m, 3)

    def pressure_force(self, patch, rho):
        F = np.zeros(3)
        _abi.check(self.lib.xcal_pressure_force(self.ctx, self.mesh.boundary_index(patch) - 1, float(rho),
                                                _abi.dptr(F)), self.ctx, "xcal_pressure_force")
        return F

    def viscous_force(self, patch, rho):
        F = np.zeros(3)
        _abi.check(self.lib.xcal_viscous_force(self.ctx, self.mesh.boundary_index(patch) - 1, float(rho),
                                               _abi.dptr(F)), self.ctx, "xcal_viscous_force")
        return F

    def set_tolerance(self, tol):
        """SIMPLE stop tolerance (1e-7 as in the reference unless changed)."""
        _abi.check(self.lib.xcal_ctx_set_tolerance(self.ctx, float(tol)), self.ctx, "xcal_ctx_set_tolerance")

    def set_field(self, which, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        _abi.check(self.lib.xcal_field_set(self.ctx, which, _abi.dptr(v), len(v)), self.ctx,
                   "xcal_field_set")

    def get_field(self, which):
        v = np.zeros(self.n)
        _abi.check(self.lib.xcal_field_get(self.ctx, which, _abi.dptr(v), self.n), self.ctx,
                   "xcal_field_get")
        return v

    def permutation(self):
        perm = np.zeros(self.n, dtype=np.int64)
        _abi.check(self.lib.xcal_mesh_permutation(self.ctx, _abi.i64ptr(perm), self.n), self.ctx,
                   "xcal_mesh_permutation")
        return perm

    def exported_mesh(self):
        """The mesh in device numbering, reference layout."""
        m = self.mesh.copy()
        a = {k: getattr(m, k) for k in ("cell_faces_ptr", "cell_faces", "cell_neighbours",
                                        "cell_nsign", "face_owner", "cell_centre", "cell_volume",
                                        "face_centre", "face_normal", "face_e", "face_area",
                                        "face_delta", "face_weight", "patch_faces", "patch_cells")}
        st = self.lib.xcal_mesh_export(
            self.ctx, _abi.i64ptr(a["cell_faces_ptr"]), _abi.i64ptr(a["cell_faces"]),
            _abi.i64ptr(a["cell_neighbours"]), _abi.i64ptr(a["cell_nsign"]),
            _abi.i64ptr(a["face_owner"]), _abi.dptr(a["cell_centre"]), _abi.dptr(a["cell_volume"]),
            _abi.dptr(a["face_centre"]), _abi.dptr(a["face_normal"]), _abi.dptr(a["face_e"]),
            _abi.dptr(a["face_area"]), _abi.dptr(a["face_delta"]), _abi.dptr(a["face_weight"]),
            _abi.i64ptr(a["patch_faces"]), _abi.i64ptr(a["patch_cells"]))
        _abi.check(st, self.ctx, "xcal_mesh_export")
        return m

    def csr(self):
        nnz = np.zeros(1, dtype=np.int64)
        n = self.n
        cap = n + int(self.mesh.cell_faces_ptr[-1] - 1)
        rp = np.zeros(n + 1, dtype=np.int32)
        col = np.zeros(cap, dtype=np.int32)
        fl = np.zeros(n, dtype=np.int32)
        bl = np.zeros(n, dtype=np.int32)
        nl = np.zeros(2, dtype=np.int32)
        _abi.check(self.lib.xcal_mesh_csr(self.ctx, _abi.i64ptr(nnz), _abi.i32ptr(rp), _abi.i32ptr(col),
                                          _abi.i32ptr(fl), _abi.i32ptr(bl), _abi.i32ptr(nl)),
                   self.ctx, "xcal_mesh_csr")
        return rp, col[: int(nnz[0])], fl, bl, nl

    def run(self, iterations, piso=False, want_krylov=True):
        R = np.ones((4, iterations))
        kry = np.zeros(5 * iterations, dtype=np.int32) if want_krylov else None
        done = np.zeros(1, dtype=np.int32)
        fn = self.lib.xcal_piso_run if piso else self.lib.xcal_simple_run
        st = fn(self.ctx, iterations, _abi.dptr(R[0]), _abi.dptr(R[1]), _abi.dptr(R[2]),
                _abi.dptr(R[3]), _abi.i32ptr(kry), _abi.i32ptr(done))
        _abi.check(st, self.ctx, "xcal_piso_run" if piso else "xcal_simple_run")
        out = dict(R_ux=R[0], R_uy=R[1], R_uz=R[2], R_p=R[3], done=int(done[0]))
        if want_krylov:
            out["krylov"] = kry.reshape(iterations, 5)
        return out

    def last_ms(self):
        ms = np.zeros(1)
        self.lib.xcal_last_run_stats(self.ctx, _abi.dptr(ms), None, 0)
        return float(ms[0])

    def autotune(self, iterations=3):
        """xcal_autotune: time the launch forms on this case (fields restored),
        keep the fastest; returns the choice as a dict."""
        r = _abi.TuneResult()
        _abi.check(self.lib.xcal_autotune(self.ctx, int(iterations), C.byref(r)), self.ctx, "xcal_autotune")
        return {k: getattr(r, k) for k, _ in _abi.TuneResult._fields_ if k != "pad"}

    def last_phases(self):
        """Per-phase-class SM cycles and phase counts of the last run (context
        created with FLAG_PHASE_TIMERS): {class: (cycles, count)}."""
        n = len(_abi.PHASES)
        cyc = np.zeros(n)
        cnt = np.zeros(n, dtype=np.int64)
        _abi.check(self.lib.xcal_last_run_phases(self.ctx, n, _abi.dptr(cyc), _abi.i64ptr(cnt)), self.ctx,
                   "xcal_last_run_phases")
        return {k: (float(cyc[i]), int(cnt[i])) for i, k in enumerate(_abi.PHASES)}

    def equation(self, which):
        n = self.n
        nnz = n + int(self.mesh.cell_faces_ptr[-1] - 1)
        vals = np.zeros(nnz)
        b = np.zeros((3, n))
        _abi.check(self.lib.xcal_equation_get(self.ctx, which, _abi.dptr(vals), _abi.dptr(b[0]),
                                              _abi.dptr(b[1]), _abi.dptr(b[2])), self.ctx,
                   "xcal_equation_get")
        return vals, b


def _upload_fields(s, model):
    s.set_field(_abi.FIELD_UX, model.U.x.values)
    s.set_field(_abi.FIELD_UY, model.U.y.values)
    s.set_field(_abi.FIELD_UZ, model.U.z.values)
    s.set_field(_abi.FIELD_P, model.p.values)
    if isturbulent(model):
        t = model.turbulence
        s.set_field(_abi.FIELD_K, t.k.values)
        s.set_field(_abi.FIELD_OMEGA, t.omega.values)
        s.set_field(_abi.FIELD_NUT, t.nut.values)


def _download_fields(s, model):
    model.U.x.values[:] = s.get_field(_abi.FIELD_UX)
    model.U.y.values[:] = s.get_field(_abi.FIELD_UY)
    model.U.z.values[:] = s.get_field(_abi.FIELD_UZ)
    model.p.values[:] = s.get_field(_abi.FIELD_P)
    if isturbulent(model):
        t = model.turbulence
        t.k.values[:] = s.get_field(_abi.FIELD_K)
        t.omega.values[:] = s.get_field(_abi.FIELD_OMEGA)
        t.nut.values[:] = s.get_field(_abi.FIELD_NUT)


def _run(model, config, pref, piso, renumber, device, precision):
    case, keep = make_case(model, config, pref, precision)
    s = Solver(model.mesh, device=device, renumber=renumber)
    try:
        s.setup(case)
        _upload_fields(s, model)
        out = s.run(config["runtime"]["iterations"], piso=piso)
        _download_fields(s, model)
    finally:
        s.close()
    return out["R_ux"], out["R_uy"], out["R_p"]


def simple(model, config, resume=True, pref=None, renumber=_abi.RENUMBER_COLOR, device=0,
           precision=_abi.PREC_FP64):
    """simple!(model, config; resume, pref) -> (R_ux, R_uy, R_p); fields updated in place."""
    return _run(model, config, pref, False, renumber, device, precision)


def piso(model, config, resume=True, pref=None, renumber=_abi.RENUMBER_COLOR, device=0,
         precision=_abi.PREC_FP64):
    """piso!(model, config; resume, pref) -> (R_ux, R_uy, R_p); fields updated in place."""
    return _run(model, config, pref, True, renumber, device, precision)


def write_vtk(name, mesh, *args):
    """write_vtk(name, mesh, ("label", field)...) (src/VTK/VTK_writer.jl:22-116):
    '<name>.vtk' with the given ScalarField/VectorField cell values.  Needs the
    mesh's nodes (meshes built from UNV files carry them)."""
    lib = _abi.load()
    labels, nco, data, keep = [], [], [], []
    for label, field in args:
        if isinstance(field, VectorField):
            arr = np.ascontiguousarray(np.concatenate([field.x.values, field.y.values, field.z.values]),
                                       dtype=np.float64)
            nco.append(3)
        elif isinstance(field, ScalarField):
            arr = np.ascontiguousarray(field.values, dtype=np.float64)
            nco.append(1)
        else:
            raise TypeError('Input data should be a ScalarField or VectorField e.g. ("U", U)')
        keep.append(arr)
        labels.append(str(label).encode())
        data.append(_abi.dptr(arr))
    n = len(labels)
    lab = (C.c_char_p * max(n, 1))(*labels)
    nc = np.array(nco or [0], dtype=np.int32)
    dat = (_abi.P_d * max(n, 1))(*data)
    st = lib.xcal_vtk_write(str(name).encode(), C.byref(mesh.desc()), n, lab, _abi.i32ptr(nc), dat)
    if st == -9:
        raise _abi.XcalError("write_vtk: the mesh has no node coordinates")
    _abi.check(st, None, "xcal_vtk_write")


def model2vtk(model, name):
    """model2vtk(model, name) (VTK_writer.jl:3-20)."""
    args = [("U", model.U), ("p", model.p)]
    if isturbulent(model):
        t = model.turbulence
        args += [("k", t.k), ("omega", t.omega), ("nut", t.nut)]
    write_vtk(name, model.mesh, *args)


class Server:
    """A stream of independent cases on one GPU (xcal_serve_*): one persistent
    launch for the server's lifetime; each case is admitted when its device
    footprint fits the server's arena, laid out by host set-up threads and
    run to `tolerance` or `max_iterations` by a group of the launch's CTAs
    sized by its mesh, beside the other cases in flight.  Every case has the
    mesh dimension `dim` and runs in `precision`.  While a server exists it
    holds the GPU: other device work of the process waits until close()."""

    def __init__(self, device=0, slots=256, max_iterations=3000, tolerance=1e-6,
                 renumber=_abi.RENUMBER_COLOR, precision=_abi.PREC_MIXED, dim=2, tiles_per_cta=0,
                 max_ctas=0, setup_threads=0, device_bytes=0.0, host_bytes=0.0):
        self.lib = _abi.load()
        self.precision = precision
        cfg = _abi.ServeCfg(slots=slots, max_iterations=max_iterations, renumber=renumber, precision=precision,
                            tolerance=tolerance, dim=dim, tiles_per_cta=tiles_per_cta, max_ctas=max_ctas,
                            setup_threads=setup_threads, device_bytes=float(device_bytes),
                            host_bytes=float(host_bytes))
        h = C.c_void_p()
        _abi.check(self.lib.xcal_serve_create(device, C.byref(cfg), C.byref(h)), None, "xcal_serve_create")
        self.srv = h
        self.ncells = {}

    def submit(self, model, config, pref=None, precision=None):
        """Queue simple!(model, config; pref) with the model's current fields as
        the initial condition; returns a ticket.  The case runs in the
        server's precision (a different `precision` raises)."""
        if precision is not None and precision != self.precision:
            raise _abi.XcalError("xcal_serve_submit: the server runs every case in its own precision")
        mesh = model.mesh
        case, keep = make_case(model, config, pref, self.precision)
        n = mesh.ncells
        U = np.ascontiguousarray(np.stack([model.U.x.values, model.U.y.values, model.U.z.values]).reshape(3 * n),
                                 dtype=np.float64)
        p = np.ascontiguousarray(model.p.values, dtype=np.float64)
        t = C.c_int64()
        _abi.check(self.lib.xcal_serve_submit(self.srv, C.byref(mesh.desc()), C.byref(case), _abi.dptr(U),
                                              _abi.dptr(p), C.byref(t)), None, "xcal_serve_submit")
        self.ncells[t.value] = n
        return t.value

    def poll(self, ticket, wait_ms=0):
        """None while the case runs; then a dict with the result and fields."""
        if ticket not in self.ncells:
            raise _abi.XcalError(f"xcal_serve_poll: unknown or already collected ticket {ticket}")
        n = self.ncells[ticket]
        res = _abi.ServeResult()
        U = np.zeros(3 * n)
        p = np.zeros(n)
        st = self.lib.xcal_serve_poll(self.srv, ticket, int(wait_ms), C.byref(res), _abi.dptr(U), _abi.dptr(p))
        if st == _abi.XCAL_PENDING:
            return None
        _abi.check(st, None, "xcal_serve_poll")
        del self.ncells[ticket]
        out = {k: getattr(res, k) for k in ("status", "iterations", "converged", "ncells", "queue_ms",
                                            "setup_ms", "run_ms", "total_ms")}
        out["residual"] = list(res.residual)
        out["U"] = U.reshape(3, n)
        out["p"] = p
        return out

    def stats(self):
        st = _abi.ServeStats()
        _abi.check(self.lib.xcal_serve_stats_get(self.srv, C.byref(st)), None, "xcal_serve_stats_get")
        return {k: getattr(st, k) for k, _ in _abi.ServeStats._fields_}

    def close(self):
        if getattr(self, "srv", None):
            self.lib.xcal_serve_destroy(self.srv)
            self.srv = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
