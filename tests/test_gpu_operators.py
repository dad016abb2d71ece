"""Operator-level API (xcal_assemble, xcal_spmv, xcal_dilu, xcal_grad and the
Python DSL of xcal.operators) against the CPU oracle's restatement of the
reference's generic _discretise! / _apply_boundary_conditions!, mul!, DILU and
grad!: a user-built Laplace equation and convection-diffusion equations on a
non-orthogonal (jittered, graded) BFS mesh and a cavity, bitwise (FP64)."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import xcal as X
from xcal import _abi, cases, meshgen
from xcal import operators as op

pytestmark = pytest.mark.gpu


def _bfs():
    return X.build_mesh(cases._unv("bfs", meshgen.bfs_unv, cells_per_h=9))


def _oracle_arrays(eqn, bcs):
    terms, srcs, bc_arr, phi, pv, keep = eqn._arrays(None, 0.0, bcs, 0)
    return terms, srcs, bc_arr, keep


@pytest.mark.parametrize("renumber", [_abi.RENUMBER_NONE, _abi.RENUMBER_COLOR], ids=["none", "color"])
def test_laplace_equation_and_solve(renumber):
    mesh = _bfs()
    E = op.Equation(mesh, renumber=renumber)
    try:
        dm = mesh if renumber == _abi.RENUMBER_NONE else _export(E, mesh)
        phi = X.ScalarField(dm)
        gamma = np.ones(dm.nfaces)
        eqn = (op.Laplacian[op.Linear](gamma, phi) == op.Source(np.zeros(dm.ncells))) >> E
        bcs = (X.Dirichlet("inlet", 1.0), X.Dirichlet("outlet", 0.0), X.Neumann("wall", 0.0), X.Neumann("top", 0.0))
        # the device works in its own numbering: conditions refer to the exported mesh's patches
        E.mesh = dm
        A0, b0 = (a.copy() for a in op.discretise(eqn))
        A, b = op.apply_boundary_conditions(eqn, bcs)
        om = O.from_mesh2(dm)
        terms, srcs, bc_arr, keep = _oracle_arrays(eqn, bcs)
        oA0, ob0 = O.assemble(om, terms, 1, srcs, 1, bc_arr, 0)
        oA, ob = O.assemble(om, terms, 1, srcs, 1, bc_arr, len(bcs))
        assert np.array_equal(A0, oA0) and np.array_equal(b0, ob0)
        assert np.array_equal(A, oA) and np.array_equal(b, ob)
        # run! with CG + DILU (the matrix is negative definite, as the reference's pressure system)
        setup = X.set_solver(phi, solver=X.CgSolver, preconditioner=X.DILU(), convergence=1e-7, relax=1.0,
                             itmax=400, atol=1e-12, rtol=1e-10)
        x = op.run(eqn, setup)
        xo, its, rn = O.linear_solve(_abi.SOLVER_CG, _abi.PRECON_DILU, E.row_ptr, E.col, A, b, np.zeros(len(b)),
                                     itmax=400, atol=1e-12, rtol=1e-10)
        assert np.array_equal(x, xo)
        assert np.linalg.norm(E.spmv(x) - b) <= 1e-8 * np.linalg.norm(b)
    finally:
        E.close()


@pytest.mark.parametrize("div", [op.Upwind, op.Linear], ids=["upwind", "linear"])
def test_convection_diffusion_with_time_si_and_sources(div):
    mesh = _bfs()
    E = op.Equation(mesh)
    try:
        rng = np.random.default_rng(3)
        n, nf = mesh.ncells, mesh.nfaces
        phi = X.ScalarField(mesh, rng.random(n))
        mdot = rng.standard_normal(nf) * 1e-3
        nu = 1e-4 * (1.0 + rng.random(nf))
        si = rng.random(n)
        src = rng.standard_normal(n)
        prev = rng.random(n)
        model = (op.Time[op.Euler](phi) + op.Divergence[div](mdot, phi) - op.Laplacian[op.Linear](nu, phi)
                 + op.Si(si, phi) == op.Source(src) - op.Source(0.5 * src))
        eqn = model >> E
        bcs = (X.Dirichlet("inlet", 0.3), X.Neumann("outlet", 0.0), X.OmegaWallFunction("wall"),
               X.KWallFunction("top"))
        runtime = X.set_runtime(iterations=1, time_step=1e-3)
        op.discretise(eqn, prev, runtime)
        A, b = op.apply_boundary_conditions(eqn, bcs)
        om = O.from_mesh2(mesh)
        terms, srcs, bc_arr, phi_v, pv, keep = eqn._arrays(prev, 1e-3, bcs, 0)
        oA, ob = O.assemble(om, terms, len(model.terms), srcs, len(model.sources), bc_arr, len(bcs),
                            phi=phi.values, prev=prev, dt=1e-3)
        assert np.array_equal(A, oA) and np.array_equal(b, ob)
        # the operators on the assembled system
        x = rng.standard_normal(n)
        assert np.array_equal(E.spmv(x), O.csr_spmv(E.row_ptr, E.col, A, x))
        y, dinv = O.dilu_apply(E.row_ptr, E.col, A, x)
        assert np.array_equal(E.dilu(x), y)
    finally:
        E.close()


def test_gradient_with_boundary_conditions():
    mesh = _bfs()
    E = op.Equation(mesh)
    try:
        rng = np.random.default_rng(9)
        phi = rng.standard_normal(mesh.ncells)
        bcs = (X.Dirichlet("inlet", 2.0), X.Neumann("outlet", 0.0), X.Dirichlet("wall", -1.0), X.Neumann("top", 0.0))
        g = op.grad(E, phi, bcs)
        bc_arr = (_abi.BC * len(bcs))()
        for k, bc in enumerate(bcs):
            bc_arr[k].patch = mesh.boundary_index(bc.ID) - 1
            bc_arr[k].type = bc.type_code
            bc_arr[k].value[:] = (float(bc.value),) * 3
        go = O.grad(O.from_mesh2(mesh), phi, bc_arr, len(bcs))
        assert np.array_equal(g[:2], go[:2])
    finally:
        E.close()


def _export(E, mesh):
    """The mesh in the context's device numbering (reference layout)."""
    lib = E.lib
    m = mesh.copy()
    a = {k: getattr(m, k) for k in ("cell_faces_ptr", "cell_faces", "cell_neighbours", "cell_nsign", "face_owner",
                                    "cell_centre", "cell_volume", "face_centre", "face_normal", "face_e",
                                    "face_area", "face_delta", "face_weight", "patch_faces", "patch_cells")}
    _abi.check(lib.xcal_mesh_export(
        E.ctx, _abi.i64ptr(a["cell_faces_ptr"]), _abi.i64ptr(a["cell_faces"]), _abi.i64ptr(a["cell_neighbours"]),
        _abi.i64ptr(a["cell_nsign"]), _abi.i64ptr(a["face_owner"]), _abi.dptr(a["cell_centre"]),
        _abi.dptr(a["cell_volume"]), _abi.dptr(a["face_centre"]), _abi.dptr(a["face_normal"]),
        _abi.dptr(a["face_e"]), _abi.dptr(a["face_area"]), _abi.dptr(a["face_delta"]),
        _abi.dptr(a["face_weight"]), _abi.i64ptr(a["patch_faces"]), _abi.i64ptr(a["patch_cells"])), E.ctx)
    m._desc = None
    return m
