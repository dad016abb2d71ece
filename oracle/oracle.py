"""ctypes binding of the CPU oracle (oracle/liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / --impl
reference legs as the checker and the CPU baseline; never by the product.
The restated reference behaviour and its documented choices are described in
xcal_oracle.cpp's header.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "xcalibre_tw.jl_b200"))
from xcal import _abi  # noqa: E402  (ctypes structs of include/xcal.h)
from xcal.mesh import Mesh2  # noqa: E402

LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp = C.c_void_p
        L.orc_build_unv.argtypes = [C.c_char_p, C.c_double, C.POINTER(vp), C.c_char_p, C.c_size_t]
        L.orc_mesh_from_desc.argtypes = [C.POINTER(_abi.MeshDesc), C.POINTER(vp), C.c_char_p, C.c_size_t]
        L.orc_mesh_free.argtypes = [vp]
        L.orc_mesh_free.restype = None
        L.orc_mesh_counts.argtypes = [vp, _abi.P_i64]
        L.orc_mesh_desc.argtypes = [vp, C.POINTER(_abi.MeshDesc)]
        L.orc_mesh_patch_names.argtypes = [vp, C.c_char_p, C.c_size_t]
        L.orc_mesh_pattern.argtypes = [vp, _abi.P_i64, _abi.P_i64]
        P_d, P_i32 = _abi.P_d, _abi.P_i32
        L.orc_run.argtypes = [vp, C.POINTER(_abi.Case), C.c_int32, C.c_int32, C.c_int64,
                              P_d, P_d, P_d, P_d, P_d, P_d, P_d, P_d, P_d, P_i32, P_i32,
                              P_d, P_d, P_d, P_d, C.c_char_p, C.c_size_t]
        L.orc_linear_solve.argtypes = [C.c_int32, C.c_int32, C.c_int64, P_i32, P_i32, P_d, P_d,
                                       P_d, C.c_int32, C.c_double, C.c_double, P_i32, P_d]
        L.orc_dilu_apply.argtypes = [C.c_int64, P_i32, P_i32, P_d, P_d, P_d, P_d]
        L.orc_precon_apply.argtypes = [C.c_int32, C.c_int64, P_i32, P_i32, P_d, P_d, P_d]
        L.orc_residual.argtypes = [C.c_int64, P_i32, P_i32, P_d, P_d, P_d]
        L.orc_residual.restype = C.c_double
        L.orc_canon_dot.argtypes = [C.c_int64, P_d, P_d]
        L.orc_canon_dot.restype = C.c_double
        L.orc_levels.argtypes = [C.c_int64, P_i32, P_i32, P_i32, P_i32]
        L.orc_renumber.argtypes = [vp, C.c_int32, _abi.P_i64]
        L.orc_last_loop_seconds.argtypes = []
        L.orc_last_loop_seconds.restype = C.c_double
        L.orc_assemble.argtypes = [vp, C.POINTER(_abi.Term), C.c_int32, C.POINTER(_abi.Source), C.c_int32,
                                   C.POINTER(_abi.BC), C.c_int32, C.c_int32, P_d, P_d, C.c_double, P_d, P_d]
        L.orc_csr_spmv.argtypes = [C.c_int64, P_i32, P_i32, P_d, P_d, P_d]
        L.orc_grad.argtypes = [vp, P_d, C.POINTER(_abi.BC), C.c_int32, P_d]
        _lib = L
    return _lib


class OracleMesh:
    def __init__(self, handle):
        self.h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle

    def __del__(self):
        try:
            if self.h:
                lib().orc_mesh_free(self.h)
        except Exception:
            pass

    def counts(self):
        c = np.zeros(8, dtype=np.int64)
        lib().orc_mesh_counts(self.h, _abi.i64ptr(c))
        return c

    def to_mesh2(self):
        d = _abi.MeshDesc()
        lib().orc_mesh_desc(self.h, C.byref(d))
        c = self.counts()
        buf = C.create_string_buffer(int(c[7]) + 16)
        lib().orc_mesh_patch_names(self.h, buf, len(buf))
        names = [s for s in buf.value.decode().split("\n") if s]
        return Mesh2.from_desc(d, names)

    def pattern(self):
        c = self.counts()
        n, tot = int(c[0]), int(c[3])
        colptr = np.zeros(n + 1, dtype=np.int64)
        rowval = np.zeros(n + tot, dtype=np.int64)
        lib().orc_mesh_pattern(self.h, _abi.i64ptr(colptr), _abi.i64ptr(rowval))
        return colptr, rowval[: colptr[-1]]

    def renumber(self, mode):
        n = int(self.counts()[0])
        perm = np.zeros(n, dtype=np.int64)
        lib().orc_renumber(self.h, mode, _abi.i64ptr(perm))
        return perm


def build_unv(path, scale=1.0):
    h = C.c_void_p()
    err = C.create_string_buffer(512)
    st = lib().orc_build_unv(str(path).encode(), scale, C.byref(h), err, 512)
    if st:
        raise RuntimeError(f"oracle build_mesh failed ({st}): {err.value.decode()}")
    return OracleMesh(h)


def from_mesh2(m):
    h = C.c_void_p()
    err = C.create_string_buffer(512)
    d = m.desc()
    st = lib().orc_mesh_from_desc(C.byref(d), C.byref(h), err, 512)
    if st:
        raise RuntimeError(f"oracle mesh import failed ({st}): {err.value.decode()}")
    return OracleMesh(h)


def run(omesh, case, iterations, U, p, k=None, omega=None, nut=None, piso=False, ref_cell=0,
        want_eqns=False):
    """Run the restated simple!/piso!.  case: xcal.api-built _abi.Case (with its
    BC arrays kept alive by the caller).  Returns a dict of results."""
    n = int(omesh.counts()[0])
    nnz = int(omesh.counts()[3]) + n
    U = np.ascontiguousarray(U, dtype=np.float64).reshape(3 * n).copy()
    p = np.ascontiguousarray(p, dtype=np.float64).copy()
    z = np.zeros(n)
    k = z.copy() if k is None else np.asarray(k, dtype=np.float64).copy()
    omega = z.copy() if omega is None else np.asarray(omega, dtype=np.float64).copy()
    nut = z.copy() if nut is None else np.asarray(nut, dtype=np.float64).copy()
    R = np.ones((4, iterations))
    kry = np.zeros(5 * iterations, dtype=np.int32)
    done = np.zeros(1, dtype=np.int32)
    AU = np.zeros(nnz) if want_eqns else None
    bU = np.zeros(3 * n) if want_eqns else None
    Ap = np.zeros(nnz) if want_eqns else None
    bp = np.zeros(n) if want_eqns else None
    err = C.create_string_buffer(512)
    st = lib().orc_run(omesh.h, C.byref(case), int(piso), iterations, ref_cell,
                       _abi.dptr(U), _abi.dptr(p), _abi.dptr(k), _abi.dptr(omega), _abi.dptr(nut),
                       _abi.dptr(R[0]), _abi.dptr(R[1]), _abi.dptr(R[2]), _abi.dptr(R[3]),
                       _abi.i32ptr(kry), _abi.i32ptr(done), _abi.dptr(AU), _abi.dptr(bU),
                       _abi.dptr(Ap), _abi.dptr(bp), err, 512)
    if st:
        raise RuntimeError(f"oracle run failed ({st}): {err.value.decode()}")
    out = dict(U=U.reshape(3, n), p=p, k=k, omega=omega, nut=nut, R_ux=R[0], R_uy=R[1],
               R_uz=R[2], R_p=R[3], krylov=kry.reshape(iterations, 5), done=int(done[0]),
               loop_seconds=float(lib().orc_last_loop_seconds()))
    if want_eqns:
        out.update(AU=AU, bU=bU.reshape(3, n), Ap=Ap, bp=bp)
    return out


def linear_solve(solver, precon, row_ptr, col, val, b, x0, itmax=100, atol=1.4901161193847656e-08,
                 rtol=1e-3):
    n = len(b)
    x = np.array(x0, dtype=np.float64).copy()
    it = np.zeros(1, dtype=np.int32)
    rn = np.zeros(1)
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cl = np.ascontiguousarray(col, dtype=np.int32)
    vv = np.ascontiguousarray(val, dtype=np.float64)
    bb = np.ascontiguousarray(b, dtype=np.float64)
    lib().orc_linear_solve(solver, precon, n, _abi.i32ptr(rp), _abi.i32ptr(cl), _abi.dptr(vv),
                           _abi.dptr(bb), _abi.dptr(x), itmax, atol, rtol, _abi.i32ptr(it),
                           _abi.dptr(rn))
    return x, int(it[0]), float(rn[0])


def precon_apply(precon, row_ptr, col, val, b):
    """y = M^{-1} b for a CSR matrix (update_preconditioner! then ldiv!)."""
    n = len(b)
    y = np.zeros(n)
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cl = np.ascontiguousarray(col, dtype=np.int32)
    vv = np.ascontiguousarray(val, dtype=np.float64)
    bb = np.ascontiguousarray(b, dtype=np.float64)
    lib().orc_precon_apply(precon, n, _abi.i32ptr(rp), _abi.i32ptr(cl), _abi.dptr(vv), _abi.dptr(bb),
                           _abi.dptr(y))
    return y


def dilu_apply(row_ptr, col, val, b):
    n = len(b)
    y = np.zeros(n)
    dinv = np.zeros(n)
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cl = np.ascontiguousarray(col, dtype=np.int32)
    vv = np.ascontiguousarray(val, dtype=np.float64)
    bb = np.ascontiguousarray(b, dtype=np.float64)
    lib().orc_dilu_apply(n, _abi.i32ptr(rp), _abi.i32ptr(cl), _abi.dptr(vv), _abi.dptr(bb),
                         _abi.dptr(y), _abi.dptr(dinv))
    return y, dinv


def canon_dot(x, y):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    return lib().orc_canon_dot(len(x), _abi.dptr(x), _abi.dptr(y))


def levels(row_ptr, col):
    n = len(row_ptr) - 1
    fl = np.zeros(n, dtype=np.int32)
    bl = np.zeros(n, dtype=np.int32)
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cl = np.ascontiguousarray(col, dtype=np.int32)
    lib().orc_levels(n, _abi.i32ptr(rp), _abi.i32ptr(cl), _abi.i32ptr(fl), _abi.i32ptr(bl))
    return fl, bl


def residual(row_ptr, col, val, x, b):
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cl = np.ascontiguousarray(col, dtype=np.int32)
    vv = np.ascontiguousarray(val, dtype=np.float64)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    bb = np.ascontiguousarray(b, dtype=np.float64)
    return lib().orc_residual(len(bb), _abi.i32ptr(rp), _abi.i32ptr(cl), _abi.dptr(vv), _abi.dptr(xx),
                              _abi.dptr(bb))


def renumbered(mesh, mode):
    """The mesh in the numbering the device uses for `mode` (0 none, 1 RCM,
    2 colour), built here from the oracle's own permutation (orc_renumber) and
    numpy, without the product library.  Rules of the renumbered layout:
    cells in new order; boundary faces keep their ids; internal faces sorted by
    (lower new owner, higher new owner, old id); every face keeps its owner
    pair orientation (owners mapped); each cell's face list ordered by new face
    id (stable); patch faces and cells mapped.  Returns (mesh, perm) with
    perm[old] = new, 0-based."""
    om = from_mesh2(mesh)
    perm = om.renumber(mode) if mode else np.arange(mesh.ncells, dtype=np.int64)
    if mode == 0:
        return mesh.copy(), perm
    nc, nf, nbf = mesh.ncells, mesh.nfaces, mesh.nbfaces
    inv = np.empty(nc, dtype=np.int64)
    inv[perm] = np.arange(nc)
    own = mesh.face_owner.reshape(nf, 2) - 1
    po = perm[own]
    fperm = np.arange(nf, dtype=np.int64)
    if nf > nbf:
        ids = np.arange(nbf, nf)
        lo = np.minimum(po[nbf:, 0], po[nbf:, 1])
        hi = np.maximum(po[nbf:, 0], po[nbf:, 1])
        order = np.lexsort((ids, hi, lo))
        fperm[ids[order]] = nbf + np.arange(nf - nbf)
    finv = np.empty(nf, dtype=np.int64)
    finv[fperm] = np.arange(nf)
    m = mesh.copy()
    m.cell_centre = np.ascontiguousarray(mesh.cell_centre.reshape(nc, 3)[inv].reshape(-1))
    m.cell_volume = np.ascontiguousarray(mesh.cell_volume[inv])
    m.face_owner = np.ascontiguousarray((po[finv] + 1).reshape(-1))
    for k in ("face_centre", "face_normal", "face_e"):
        setattr(m, k, np.ascontiguousarray(getattr(mesh, k).reshape(nf, 3)[finv].reshape(-1)))
    for k in ("face_area", "face_delta", "face_weight"):
        setattr(m, k, np.ascontiguousarray(getattr(mesh, k)[finv]))
    ptr = mesh.cell_faces_ptr - 1
    cnt = np.diff(ptr)[inv]
    nptr = np.concatenate([[0], np.cumsum(cnt)])
    src = np.repeat(ptr[inv] - nptr[:-1], cnt) + np.arange(nptr[-1])
    owner_of = np.repeat(np.arange(nc), cnt)
    newf = fperm[mesh.cell_faces[src] - 1]
    order = np.lexsort((newf, owner_of))        # stable by new face id inside each cell
    src = src[order]
    m.cell_faces_ptr = np.ascontiguousarray(nptr + 1)
    m.cell_faces = np.ascontiguousarray(fperm[mesh.cell_faces[src] - 1] + 1)
    m.cell_neighbours = np.ascontiguousarray(perm[mesh.cell_neighbours[src] - 1] + 1)
    m.cell_nsign = np.ascontiguousarray(mesh.cell_nsign[src])
    m.patch_faces = np.ascontiguousarray(fperm[mesh.patch_faces - 1] + 1)
    m.patch_cells = np.ascontiguousarray(perm[mesh.patch_cells - 1] + 1)
    if m.nnodes > 0:
        cnp = mesh.cell_nodes_ptr - 1
        nn = np.diff(cnp)[inv]
        nnp = np.concatenate([[0], np.cumsum(nn)])
        m.cell_nodes_ptr = np.ascontiguousarray(nnp + 1)
        m.cell_nodes = np.ascontiguousarray(mesh.cell_nodes[np.repeat(cnp[inv] - nnp[:-1], nn) + np.arange(nnp[-1])])
    m._desc = None
    return m, perm


def assemble(omesh, terms, nterms, sources, nsources, bcs, nbc, component=0, phi=None, prev=None, dt=0.0):
    """Generic discretise! (+ apply_boundary_conditions! with nbc > 0) of a model
    equation given as ctypes arrays of xcal_term / xcal_source / xcal_bc;
    returns (CSR values in the pattern's order, b)."""
    c = omesh.counts()
    n, tot = int(c[0]), int(c[3])
    vals = np.zeros(n + tot)
    b = np.zeros(n)
    st = lib().orc_assemble(omesh.h, terms, nterms, sources, nsources, bcs, nbc, component,
                            _abi.dptr(None if phi is None else np.ascontiguousarray(phi, dtype=np.float64)),
                            _abi.dptr(None if prev is None else np.ascontiguousarray(prev, dtype=np.float64)),
                            float(dt), _abi.dptr(vals), _abi.dptr(b))
    if st:
        raise RuntimeError(f"oracle assemble failed ({st})")
    return vals, b


def csr_spmv(row_ptr, col, val, x):
    n = len(row_ptr) - 1
    y = np.zeros(n)
    lib().orc_csr_spmv(n, _abi.i32ptr(np.ascontiguousarray(row_ptr, dtype=np.int32)),
                       _abi.i32ptr(np.ascontiguousarray(col, dtype=np.int32)),
                       _abi.dptr(np.ascontiguousarray(val, dtype=np.float64)),
                       _abi.dptr(np.ascontiguousarray(x, dtype=np.float64)), _abi.dptr(y))
    return y


def grad(omesh, phi, bcs, nbc):
    n = int(omesh.counts()[0])
    g = np.zeros(3 * n)
    st = lib().orc_grad(omesh.h, _abi.dptr(np.ascontiguousarray(phi, dtype=np.float64)), bcs, nbc, _abi.dptr(g))
    if st:
        raise RuntimeError(f"oracle grad failed ({st})")
    return g.reshape(3, n)
