"""The reference's operator-level API (module ModelFramework, Discretise):
user-built model equations, discretised and solved on the GPU.

    model = (Time[Euler](phi) + Divergence[Upwind](mdotf, phi)
             - Laplacian[Linear](gamma, phi) == Source(src))      # Model
    eqn = model >> Equation(mesh)                                  # the reference's `→`
    discretise(eqn, prev, runtime)                                 # discretise!
    apply_boundary_conditions(eqn, (Dirichlet("inlet", 1.0), ...)) # apply_boundary_conditions!
    x = run(eqn, setup, x0)                                        # run!

Operators (src/ModelFramework/ModelFramework_0_types.jl:15-81): Time{Steady|Euler},
Laplacian{Linear}, Divergence{Linear|Upwind}, Si (implicit source) take a face
flux field (one value per face; Si: per cell) and the field they act on;
Source(field) is an explicit cell source.  `+`, `-` (the second operand's
sign becomes -1) and `==` follow ModelFramework_1_operations.jl:3-58.  Python
has no `→`, so `model >> Equation(mesh)` binds a model to its equation.

Fields are in the numbering of the equation's device context (the caller's
own with renumber=RENUMBER_NONE, the default here).  The equation's matrix
comes back in CSR (row) order of eqn.row_ptr / eqn.col.
"""
import ctypes as C

import numpy as np

from . import _abi
from .api import Linear, Steady, Euler, Upwind, _BC  # noqa: F401


class _Scheme:
    """Operator[Scheme](...) as Operator{Scheme}(...) in Julia."""

    def __init__(self, op, scheme):
        self.op, self.scheme = op, scheme

    def __call__(self, *args):
        o = self.op(*args)
        o.scheme = self.scheme
        return o


class Operator:
    kind = None
    default_scheme = None

    def __init__(self, flux, phi):
        self.flux = flux
        self.phi = phi
        self.sign = 1.0
        self.scheme = self.default_scheme

    def __class_getitem__(cls, scheme):
        return _Scheme(cls, scheme)

    def _neg(self):
        o = object.__new__(type(self))
        o.__dict__.update(self.__dict__)
        o.sign = -1.0
        return o

    def __add__(self, other):
        return _terms(self) + _terms(other)

    def __radd__(self, other):
        return _terms(other) + _terms(self)

    def __sub__(self, other):
        return _terms(self) + [t._neg() for t in _terms(other)]

    def __eq__(self, sources):
        return Model(_terms(self), _sources(sources))

    __hash__ = object.__hash__


class Time(Operator):
    kind = _abi.TERM_TIME
    default_scheme = Steady

    def __init__(self, phi):
        super().__init__(None, phi)


class Laplacian(Operator):
    kind = _abi.TERM_LAPLACIAN
    default_scheme = Linear


class Divergence(Operator):
    kind = _abi.TERM_DIVERGENCE
    default_scheme = Linear


class Si(Operator):
    kind = _abi.TERM_SI
    default_scheme = None


class Source:
    def __init__(self, field, sign=1.0):
        self.field = field
        self.sign = sign

    def __neg__(self):
        return [Source(self.field, -1.0)]

    def __add__(self, other):
        return _sources(self) + _sources(other)

    def __sub__(self, other):
        return _sources(self) + [Source(s.field, -1.0) for s in _sources(other)]


class _TermList(list):
    def __add__(self, other):
        return _TermList(list(self) + _terms(other))

    def __sub__(self, other):
        return _TermList(list(self) + [t._neg() for t in _terms(other)])

    def __eq__(self, sources):
        return Model(list(self), _sources(sources))

    __hash__ = object.__hash__


def _terms(x):
    if isinstance(x, Operator):
        return _TermList([x])
    return _TermList(list(x))


def _sources(x):
    if isinstance(x, Source):
        return [x]
    return list(x)


def _values(f):
    v = getattr(f, "values", f)
    return np.ascontiguousarray(v, dtype=np.float64)


class Model:
    """Model{terms, sources} (ModelFramework_0_types.jl:60-81)."""

    def __init__(self, terms, sources):
        if not terms:
            raise ValueError("a model needs at least one operator")
        self.terms = list(terms)
        self.sources = list(sources)

    def __rshift__(self, eqn):
        return ModelEquation(self, eqn)


class Equation:
    """Equation(mesh) (ModelFramework_0_types.jl:83-125): the sparsity pattern
    of the mesh on a device context, with A (CSR values) and b."""

    def __init__(self, mesh, renumber=_abi.RENUMBER_NONE, device=0):
        self.lib = _abi.load()
        self.mesh = mesh
        h = C.c_void_p()
        _abi.check(self.lib.xcal_ctx_create(device, 0, C.byref(h)), None, "xcal_ctx_create")
        self.ctx = h
        _abi.check(self.lib.xcal_mesh_upload(self.ctx, C.byref(mesh.desc()), renumber), self.ctx,
                   "xcal_mesh_upload")
        n = mesh.ncells
        nnz = np.zeros(1, dtype=np.int64)
        cap = n + len(mesh.cell_faces)
        rp = np.zeros(n + 1, dtype=np.int32)
        col = np.zeros(cap, dtype=np.int32)
        _abi.check(self.lib.xcal_mesh_csr(self.ctx, _abi.i64ptr(nnz), _abi.i32ptr(rp), _abi.i32ptr(col), None, None,
                                          None), self.ctx, "xcal_mesh_csr")
        self.row_ptr, self.col = rp, col[: int(nnz[0])]
        self.A = np.zeros(int(nnz[0]))
        self.b = np.zeros(n)

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.xcal_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def spmv(self, x):
        """mul!(y, A, x) on the device."""
        x = _values(x)
        y = np.zeros(len(self.b))
        _abi.check(self.lib.xcal_spmv(self.ctx, _abi.dptr(self.A), _abi.dptr(x), _abi.dptr(y)), self.ctx, "xcal_spmv")
        return y

    def dilu(self, r):
        """update_preconditioner! + ldiv! of DILU on A, on the device."""
        r = _values(r)
        y = np.zeros(len(self.b))
        _abi.check(self.lib.xcal_dilu(self.ctx, _abi.dptr(self.A), _abi.dptr(r), _abi.dptr(y)), self.ctx, "xcal_dilu")
        return y


class ModelEquation:
    """ModelEquation(model, equation) (the result of `→`)."""

    def __init__(self, model, equation):
        self.model = model
        self.equation = equation

    def _arrays(self, prev, dt, bcs, component):
        m = self.model
        keep = []
        terms = (_abi.Term * len(m.terms))()
        phi = None
        for k, t in enumerate(m.terms):
            terms[k].kind = t.kind
            terms[k].sign = t.sign
            if t.kind == _abi.TERM_TIME:
                terms[k].scheme = t.scheme.code
                terms[k].flux = None
            else:
                terms[k].scheme = t.scheme.code if t.scheme is not None else 0
                f = _values(t.flux)
                keep.append(f)
                terms[k].flux = _abi.dptr(f)
            if t.phi is not None and phi is None:
                phi = _values(t.phi)
        srcs = (_abi.Source * max(1, len(m.sources)))()
        for k, s in enumerate(m.sources):
            f = _values(s.field)
            keep.append(f)
            srcs[k].sign = s.sign
            srcs[k].field = _abi.dptr(f)
        bc_arr = (_abi.BC * max(1, len(bcs)))()
        mesh = self.equation.mesh
        for k, bc in enumerate(bcs):
            e = bc_arr[k]
            e.patch = mesh.boundary_index(bc.ID) - 1
            e.type = bc.type_code
            v = bc.value
            if isinstance(v, dict):
                v = 0.0
            if isinstance(v, (list, tuple, np.ndarray)):
                e.value[:] = (float(v[0]), float(v[1]), float(v[2]))
            else:
                e.value[:] = (float(v), float(v), float(v))
        pv = _values(prev) if prev is not None else None
        if phi is not None:
            keep.append(phi)
        if pv is not None:
            keep.append(pv)
        return terms, srcs, bc_arr, phi, pv, keep

    def assemble(self, prev=None, runtime=None, bcs=(), component=0):
        dt = float(runtime["dt"]) if runtime is not None else 0.0
        terms, srcs, bc_arr, phi, pv, keep = self._arrays(prev, dt, bcs, component)
        E = self.equation
        _abi.check(E.lib.xcal_assemble(E.ctx, terms, len(self.model.terms), srcs, len(self.model.sources), bc_arr,
                                       len(bcs), component, _abi.dptr(phi), _abi.dptr(pv), dt, _abi.dptr(E.A),
                                       _abi.dptr(E.b)), E.ctx, "xcal_assemble")
        self._last = (prev, runtime)
        return E.A, E.b


def discretise(eqn, prev=None, runtime=None):
    """discretise!(eqn, prev, runtime): A and b of the model's terms and sources."""
    eqn._bcs = ()
    return eqn.assemble(prev, runtime)


def apply_boundary_conditions(eqn, BCs, component=0):
    """apply_boundary_conditions!(eqn, BCs) after discretise!: the boundary
    contributions of every condition (in order) for every term."""
    prev, runtime = getattr(eqn, "_last", (None, None))
    return eqn.assemble(prev, runtime, tuple(BCs), component)


def run(eqn, setup, x0=None):
    """run!(eqn, setup) with the solver settings of set_solver (Krylov.jl
    solve! with warm start x0): returns the solution."""
    E = eqn.equation
    n = len(E.b)
    x = np.zeros(n) if x0 is None else np.array(_values(x0), dtype=np.float64)
    it = np.zeros(1, dtype=np.int32)
    rn = np.zeros(1)
    pc = setup["preconditioner"].code
    if pc is None:
        raise _abi.XcalError("run: preconditioner not available")
    _abi.check(E.lib.xcal_linear_solve(E.ctx, setup["solver"].code, pc, n, _abi.i32ptr(E.row_ptr),
                                       _abi.i32ptr(E.col), _abi.dptr(E.A), _abi.dptr(E.b), _abi.dptr(x),
                                       setup["itmax"], setup["atol"], setup["rtol"], _abi.i32ptr(it),
                                       _abi.dptr(rn)), E.ctx, "xcal_linear_solve")
    return x


def grad(eqn_or_equation, phi, BCs=()):
    """grad! (Orthogonal, Green-Gauss) of a cell field with its conditions:
    array (3, ncells)."""
    E = getattr(eqn_or_equation, "equation", eqn_or_equation)
    mesh = E.mesh
    phi = _values(phi)
    bc_arr = (_abi.BC * max(1, len(BCs)))()
    for k, bc in enumerate(BCs):
        e = bc_arr[k]
        e.patch = mesh.boundary_index(bc.ID) - 1
        e.type = bc.type_code
        v = bc.value if not isinstance(bc.value, dict) else 0.0
        e.value[:] = (float(v), float(v), float(v))
    g = np.zeros(3 * mesh.ncells)
    _abi.check(E.lib.xcal_grad(E.ctx, _abi.dptr(phi), bc_arr, len(BCs), _abi.dptr(g)), E.ctx, "xcal_grad")
    return g.reshape(3, mesh.ncells)
