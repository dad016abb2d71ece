"""Device (libxcal.so, sm_100a) against the CPU oracle: FP64 results must agree
to relative L2 <= 1e-10 on every residual history, field and assembled system;
Krylov iteration counts must be identical.  With the canonical reduction order
and --fmad=false the comparison is expected to be bitwise (0.0)."""
import os

import numpy as np
import pytest

import oracle as O
import xcal as X
from xcal import _abi, cases
from parity_util import TOL, assert_parity, run_device, run_oracle

pytestmark = pytest.mark.gpu

MODES = [_abi.RENUMBER_NONE, _abi.RENUMBER_RCM, _abi.RENUMBER_COLOR]


@pytest.mark.parametrize("renumber", MODES, ids=["none", "rcm", "color"])
def test_cavity_simple_parity(renumber):
    """Configuration 1: 40x40 cavity, Re=100, 1000 iterations (stops at 1e-7)."""
    mesh, model, config, pref = cases.cavity2d(40, iterations=1000)
    dev = run_device(mesh, model, config, pref, 1000, renumber)
    orc = run_oracle(dev["dev_mesh"], model, config, pref, 1000, dev["perm"])
    d = assert_parity(dev, orc)
    print("cavity", renumber, dev["done"], d)


@pytest.mark.parametrize("renumber", [_abi.RENUMBER_NONE, _abi.RENUMBER_COLOR], ids=["none", "color"])
def test_bfs_simple_parity(renumber):
    """Configuration 2 (47,385-cell jittered BFS), first 25 SIMPLE iterations."""
    mesh, model, config, pref = cases.bfs(27, iterations=25)
    dev = run_device(mesh, model, config, pref, 25, renumber)
    orc = run_oracle(dev["dev_mesh"], model, config, pref, 25, dev["perm"])
    d = assert_parity(dev, orc)
    print("bfs", renumber, d)


def test_schemes_linear_midpoint():
    """Divergence{Linear} and the Midpoint gradient on a coarse jittered BFS."""
    mesh, model, config, pref = cases.bfs(6, iterations=60, divergence=X.Linear, gradient=X.Midpoint)
    dev = run_device(mesh, model, config, pref, 60, _abi.RENUMBER_COLOR)
    orc = run_oracle(dev["dev_mesh"], model, config, pref, 60, dev["perm"])
    assert_parity(dev, orc)


def test_solver_preconditioner_variants():
    """BiCGSTAB for p and the Jacobi / NormDiagonal / no preconditioners."""
    for precon, p_solver in ((X.Jacobi, X.BicgstabSolver), (X.NormDiagonal, X.CgSolver), (X.DILU, X.BicgstabSolver)):
        mesh, model, config, pref = cases.cavity2d(24, iterations=40, precon=precon, p_solver=p_solver)
        dev = run_device(mesh, model, config, pref, 40, _abi.RENUMBER_RCM)
        orc = run_oracle(dev["dev_mesh"], model, config, pref, 40, dev["perm"])
        assert_parity(dev, orc)


def test_piso_parity():
    """piso! with the Euler time term: 2 correctors per step, no relaxation of U."""
    mesh, model, config, pref = cases.cavity2d(32, iterations=15)
    config["schemes"]["U"] = X.set_schemes(time=X.Euler, divergence=X.Upwind)
    config["runtime"] = X.set_runtime(iterations=15, write_interval=-1, time_step=1e-3)
    dev = run_device(mesh, model, config, pref, 15, _abi.RENUMBER_COLOR, piso=True)
    orc = run_oracle(dev["dev_mesh"], model, config, pref, 15, dev["perm"], piso=True)
    assert_parity(dev, orc)


def test_hex_cavity_parity():
    """3D extension (uz equation, hexahedra): 12^3 cavity, 20 iterations."""
    mesh, model, config, pref = cases.cavity3d(12, iterations=20)
    dev = run_device(mesh, model, config, pref, 20, _abi.RENUMBER_COLOR)
    orc = run_oracle(dev["dev_mesh"], model, config, pref, 20, dev["perm"])
    assert_parity(dev, orc, nU=3)


@pytest.mark.parametrize("sync", ["block", "cluster", "grid"])
def test_barrier_modes_identical(sync, monkeypatch):
    """The result does not depend on how many CTAs run the program."""
    monkeypatch.setenv("XCAL_SYNC", sync)
    mesh, model, config, pref = cases.cavity2d(20, iterations=30)
    dev = run_device(mesh, model, config, pref, 30, _abi.RENUMBER_COLOR)
    monkeypatch.delenv("XCAL_SYNC")
    ref = run_device(mesh, model, config, pref, 30, _abi.RENUMBER_COLOR)
    for k in ("R_ux", "R_uy", "R_p", "p"):
        assert np.array_equal(np.nan_to_num(dev[k], nan=-1), np.nan_to_num(ref[k], nan=-1)), k
    assert np.array_equal(dev["U"], ref["U"])


@pytest.mark.parametrize("fuse", ["0", "1"], ids=["cg3", "cg2"])
def test_cg_fused_and_split_phases(fuse, monkeypatch):
    """CG with the two-level DILU applied inside the x/r phase (2 grid
    barriers per iteration) and with a separate backward phase (3 barriers):
    both agree bitwise with the oracle, on 2D and 3D meshes."""
    monkeypatch.setenv("XCAL_CG_FUSE", fuse)
    mesh, model, config, pref = cases.bfs(6, iterations=40)
    dev = run_device(mesh, model, config, pref, 40, _abi.RENUMBER_COLOR)
    orc = run_oracle(dev["dev_mesh"], model, config, pref, 40, dev["perm"])
    assert_parity(dev, orc)
    mesh, model, config, pref = cases.cavity3d(10, iterations=15)
    dev = run_device(mesh, model, config, pref, 15, _abi.RENUMBER_COLOR)
    orc = run_oracle(dev["dev_mesh"], model, config, pref, 15, dev["perm"])
    assert_parity(dev, orc, nU=3)


@pytest.mark.parametrize("occ", ["2", "4"])
def test_occupancy_builds_match_oracle(occ, monkeypatch):
    """The 2-CTA/SM and 4-CTA/SM builds of the persistent program (forced
    with XCAL_OCC, grid barrier) compute the same values: bitwise equal to the
    oracle on the 2D BFS and the 3D cavity, FP64."""
    monkeypatch.setenv("XCAL_OCC", occ)
    monkeypatch.setenv("XCAL_SYNC", "grid")
    mesh, model, config, pref = cases.bfs(6, iterations=30)
    dev = run_device(mesh, model, config, pref, 30, _abi.RENUMBER_COLOR)
    orc = run_oracle(dev["dev_mesh"], model, config, pref, 30, dev["perm"])
    assert_parity(dev, orc)
    mesh, model, config, pref = cases.cavity3d(12, iterations=10)
    dev = run_device(mesh, model, config, pref, 10, _abi.RENUMBER_COLOR)
    orc = run_oracle(dev["dev_mesh"], model, config, pref, 10, dev["perm"])
    assert_parity(dev, orc, nU=3)


def test_grid_barrier_repeatable(monkeypatch):
    """The grid barrier's acquire/release ordering under load: 100 SIMPLE
    iterations of the full 47,385-cell BFS (about 33,000 grid barriers) give
    bitwise identical histories and fields run twice with the default grid,
    and with 93 CTAs of two tiles each."""
    mesh, model, config, pref = cases.bfs(27, iterations=100)
    runs = [run_device(mesh, model, config, pref, 100, _abi.RENUMBER_COLOR) for _ in range(2)]
    monkeypatch.setenv("XCAL_SYNC", "grid")
    monkeypatch.setenv("XCAL_NBLOCKS", "93")
    runs.append(run_device(mesh, model, config, pref, 100, _abi.RENUMBER_COLOR))
    ref = runs[0]
    for r in runs[1:]:
        for k in ("R_ux", "R_uy", "R_p"):
            assert np.array_equal(np.nan_to_num(r[k], nan=-1), np.nan_to_num(ref[k], nan=-1)), k
        assert np.array_equal(r["U"], ref["U"]) and np.array_equal(r["p"], ref["p"])
        assert np.array_equal(r["krylov"], ref["krylov"])


def _snapshot_matrix(n=24, iters=5):
    mesh, model, config, pref = cases.cavity2d(n, iterations=iters)
    om = O.from_mesh2(mesh)
    case, keep = X.make_case(model, config, pref)
    U, p = cases.fields(model)
    out = O.run(om, case, iters, U, p, want_eqns=True)
    colptr, rowval = om.pattern()
    return colptr.astype(np.int32), rowval.astype(np.int32), out


@pytest.mark.parametrize("solver", [_abi.SOLVER_CG, _abi.SOLVER_BICGSTAB, _abi.SOLVER_GMRES],
                         ids=["cg", "bicgstab", "gmres"])
@pytest.mark.parametrize("precon", [_abi.PRECON_DILU, _abi.PRECON_ILU0, _abi.PRECON_JACOBI, _abi.PRECON_NONE],
                         ids=["dilu", "ilu0", "jacobi", "none"])
@pytest.mark.parametrize("matrix", ["Ap", "AU"])
def test_linear_solve_parity(solver, precon, matrix):
    """run! on a standalone CSR system: the cavity's pressure matrix (symmetric)
    and its momentum matrix (upwind convection, nonsymmetric)."""
    if solver == _abi.SOLVER_CG and matrix == "AU":
        pytest.skip("CG needs a symmetric system")
    rp, col, out = _snapshot_matrix()
    A = out[matrix]
    n = len(rp) - 1
    rng = np.random.default_rng(7)
    b = rng.standard_normal(n)
    x0 = rng.standard_normal(n) * 0.1
    xo, ito, rno = O.linear_solve(solver, precon, rp, col, A, b, x0, itmax=200, rtol=1e-8)
    lib = _abi.load()
    import ctypes as C
    h = C.c_void_p()
    _abi.check(lib.xcal_ctx_create(0, 0, C.byref(h)))
    try:
        x = x0.copy()
        it = np.zeros(1, dtype=np.int32)
        rn = np.zeros(1)
        _abi.check(lib.xcal_linear_solve(h, solver, precon, n, _abi.i32ptr(rp), _abi.i32ptr(col),
                                         _abi.dptr(A), _abi.dptr(b), _abi.dptr(x), 200,
                                         1.4901161193847656e-08, 1e-8, _abi.i32ptr(it), _abi.dptr(rn)), h)
    finally:
        lib.xcal_ctx_destroy(h)
    assert int(it[0]) == ito
    assert np.linalg.norm(x - xo) <= TOL * np.linalg.norm(xo)
    assert rn[0] == rno or abs(rn[0] - rno) <= TOL * abs(rno)


@pytest.mark.parametrize("u_solver,p_solver,precon", [
    (X.GmresSolver, X.CgSolver, X.ILU0),
    (X.GmresSolver, X.GmresSolver, X.DILU),
    (X.BicgstabSolver, X.CgSolver, X.ILU0),
], ids=["gmres-ilu0", "gmres-gmres-dilu", "bicgstab-cg-ilu0"])
def test_gmres_ilu0_simple_parity(u_solver, p_solver, precon):
    """simple! with GmresSolver and ILU0() as in the reference's case scripts
    (CASE_UNV_BFS.jl, CASE_cylinder_U.jl): 30 iterations on a jittered BFS."""
    mesh, model, config, pref = cases.bfs(5, iterations=30, u_solver=u_solver, p_solver=p_solver, precon=precon)
    dev = run_device(mesh, model, config, pref, 30, _abi.RENUMBER_COLOR)
    orc = run_oracle(dev["dev_mesh"], model, config, pref, 30, dev["perm"])
    assert_parity(dev, orc)


def test_field_roundtrip_and_permutation():
    mesh, model, config, pref = cases.bfs(6, iterations=1)
    case, keep = X.make_case(model, config, pref)
    s = X.Solver(mesh, renumber=_abi.RENUMBER_COLOR)
    try:
        s.setup(case)
        v = np.arange(mesh.ncells, dtype=np.float64) * 0.5 - 3.0
        for f in (_abi.FIELD_UX, _abi.FIELD_UY, _abi.FIELD_UZ, _abi.FIELD_P):
            s.set_field(f, v + f)
        for f in (_abi.FIELD_UX, _abi.FIELD_UY, _abi.FIELD_UZ, _abi.FIELD_P):
            assert np.array_equal(s.get_field(f), v + f)
        perm = s.permutation()
        assert np.array_equal(np.sort(perm), np.arange(1, mesh.ncells + 1))
    finally:
        s.close()


def test_api_simple_end_to_end():
    """The reference-shaped API: simple(model, config; pref) updates fields in place."""
    mesh, model, config, pref = cases.cavity2d(16, iterations=50)
    Rx, Ry, Rp = X.simple(model, config, pref=pref)
    assert len(Rx) == 50 and np.isnan(Ry[0])   # 0/0 in the first uy residual, as in the reference
    assert np.all(np.isfinite(model.p.values)) and np.abs(model.U.x.values).max() > 0.1


def test_residual_operator_parity():
    """xcal_residual (residual! on a CSR system) against the oracle."""
    import ctypes as C
    rp, col, out = _snapshot_matrix(n=30, iters=4)
    A = out["Ap"]
    n = len(rp) - 1
    rng = np.random.default_rng(3)
    x = rng.standard_normal(n)
    b = rng.standard_normal(n)
    ro = O.residual(rp, col, A, x, b)
    lib = _abi.load()
    h = C.c_void_p()
    _abi.check(lib.xcal_ctx_create(0, 0, C.byref(h)))
    try:
        R = np.zeros(1)
        _abi.check(lib.xcal_residual(h, n, _abi.i32ptr(rp), _abi.i32ptr(col), _abi.dptr(A), _abi.dptr(x),
                                     _abi.dptr(b), _abi.dptr(R)), h)
    finally:
        lib.xcal_ctx_destroy(h)
    assert R[0] == ro or abs(R[0] - ro) <= TOL * abs(ro)


def test_komega_flatplate_parity():
    """k-omega (turbulence!, omega wall function) on a coarse graded flat plate."""
    mesh, model, config, pref = cases.flatplate(60, 30, iterations=40)
    dev = run_device(mesh, model, config, pref, 40, _abi.RENUMBER_COLOR)
    orc = run_oracle(dev["dev_mesh"], model, config, pref, 40, dev["perm"])
    d = assert_parity(dev, orc)
    print("komega", d)


def test_komega_wall_functions_parity():
    """k and nut wall functions (correct_production!, correct_nut_wall!): their
    log() comes from CUDA on the device and from libm in the oracle, so the
    comparison uses the FP64 tolerance rather than bit equality."""
    mesh, model, config, pref = cases.flatplate(60, 30, iterations=30, wall_functions=True)
    dev = run_device(mesh, model, config, pref, 30, _abi.RENUMBER_COLOR)
    orc = run_oracle(dev["dev_mesh"], model, config, pref, 30, dev["perm"])
    d = assert_parity(dev, orc)
    print("komega-wf", d)
