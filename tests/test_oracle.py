"""The CPU oracle against what pins it: the reference's own mesh fixtures
(counts by hand), known-answer problems and structural invariants.  There is no
Julia here and the reference ships no golden vectors for this path, so FP
parity with the reference's own run is unpinned; tests/golden holds the
oracle's own regression vectors (generated by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import oracle as O
import xcal as X
from xcal import _abi, cases, meshgen

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_quad40_reference_fixture(ref_meshes):
    m = O.build_unv(os.path.join(ref_meshes, "quad40.unv"), scale=0.001)
    c = m.counts()
    assert (c[0], c[1], c[2]) == (1600, 3280, 160)     # 40x40 quads, 2*40*41 edges, 4*40 boundary
    M = m.to_mesh2()
    assert M.patch_names == ["inlet", "outlet", "bottom", "top"]
    assert abs(M.cell_volume.sum() - 1.0) < 1e-12        # 1000 mm square scaled to 1 m


@pytest.mark.parametrize("name,cells,faces,bfaces", [
    ("quad.unv", None, None, None), ("trig40.unv", None, None, None),
    ("backwardFacingStep_10mm.unv", 1800, 3720, 240)])
def test_reference_meshes_invariants(ref_meshes, name, cells, faces, bfaces):
    M = O.build_unv(os.path.join(ref_meshes, name), scale=0.001).to_mesh2()
    if cells:
        assert (M.ncells, M.nfaces, M.nbfaces) == (cells, faces, bfaces)
    _check_invariants(M)


def _check_invariants(M):
    n = M.ncells
    ptr = M.cell_faces_ptr - 1
    # Euler: every internal face listed twice with opposite nsign
    assert len(M.cell_faces) == 2 * (M.nfaces - M.nbfaces)
    own = M.face_owner.reshape(-1, 2) - 1
    assert np.all(own[: M.nbfaces, 0] == own[: M.nbfaces, 1])
    assert np.all(own[M.nbfaces:, 0] < own[M.nbfaces:, 1])
    # closed cells: sum over faces of nsign * area * normal = 0
    S = np.zeros((n, 3))
    nrm = M.face_normal.reshape(-1, 3)
    for c in range(n):
        for k in range(ptr[c], ptr[c + 1]):
            f = M.cell_faces[k] - 1
            S[c] += M.cell_nsign[k] * M.face_area[f] * nrm[f]
    for f in range(M.nbfaces):
        S[own[f, 0]] += M.face_area[f] * nrm[f]
    assert np.abs(S).max() < 1e-9 * M.face_area.max()
    assert np.all(M.cell_volume > 0)


def test_generated_meshes_invariants():
    for fn, kw in ((meshgen.cavity_unv, dict(n=12, L=0.1)), (meshgen.bfs_unv, dict(cells_per_h=5)),
                   (meshgen.flatplate_unv, dict(nx=30, ny=20))):
        path = f"/tmp/xcal_inv_{fn.__name__}.unv"
        fn(path, **kw)
        M = O.build_unv(path).to_mesh2()
        _check_invariants(M)
    M = X.Mesh2.from_dict(meshgen.hex_cavity(6))
    assert abs(M.cell_volume.sum() - 1.0) < 1e-12
    O.from_mesh2(M)   # the oracle accepts the 3D layout


def test_bfs_configuration_size():
    path = cases._unv("bfs", meshgen.bfs_unv, cells_per_h=27)
    M = O.build_unv(path).to_mesh2()
    assert (M.ncells, M.nfaces - M.nbfaces, M.nbfaces) == (47385, 93771, 1998)
    assert abs(M.cell_volume.sum() - 0.0065) < 1e-12


def test_laplace_known_answer():
    """Uniform orthogonal mesh, Laplacian with Dirichlet ends: the linear profile
    is the exact discrete solution (dynamic_proto_operators.jl:76-85,225-229)."""
    path = "/tmp/xcal_laplace.unv"
    meshgen.cavity_unv(path, n=10, L=1.0)
    M = O.build_unv(path).to_mesh2()
    colptr, rowval = O.from_mesh2(M).pattern()
    n = M.ncells
    # assemble -Laplacian(1, T) with T=0 at inlet (x=0), T=1 at outlet (x=1)
    ptr = M.cell_faces_ptr - 1
    A = {}
    b = np.zeros(n)
    for c in range(n):
        A[(c, c)] = 0.0
        for k in range(ptr[c], ptr[c + 1]):
            f = M.cell_faces[k] - 1
            nb = M.cell_neighbours[k] - 1
            ap = M.face_area[f] / M.face_delta[f]
            A[(c, c)] += ap
            A[(c, nb)] = A.get((c, nb), 0.0) - ap
    for name, val in (("inlet", 0.0), ("outlet", 1.0)):
        i = M.patch_names.index(name)
        for k in range(M.patch_ptr[i], M.patch_ptr[i + 1]):
            f, c = M.patch_faces[k] - 1, M.patch_cells[k] - 1
            ap = M.face_area[f] / M.face_delta[f]
            A[(c, c)] += ap
            b[c] += ap * val
    vals = np.array([A[(r, int(rowval[q]))] for r in range(n) for q in range(colptr[r], colptr[r + 1])])
    x, it, rn = O.linear_solve(_abi.SOLVER_CG, _abi.PRECON_DILU, colptr.astype(np.int32),
                               rowval.astype(np.int32), vals, b, np.zeros(n), itmax=200, atol=1e-14,
                               rtol=1e-14)
    xc = M.cell_centre.reshape(-1, 3)[:, 0]
    assert np.abs(x - xc).max() < 1e-10


def test_canonical_sum_order():
    """The canonical reduction is exact on integers and differs from naive
    summation only by rounding."""
    x = np.arange(5000, dtype=np.float64)
    assert O.canon_dot(x, np.ones_like(x)) == x.sum()
    rng = np.random.default_rng(0)
    a, b = rng.standard_normal(12345), rng.standard_normal(12345)
    assert abs(O.canon_dot(a, b) - float(a @ b)) < 1e-10


def test_cavity_oracle_behaviour():
    """Reference behaviours kept by the restatement: R_uy[1] is 0/0 (b_y = 0),
    histories stop at 1e-7 with trailing 1.0, and the lid drives a vortex."""
    mesh, model, config, pref = cases.cavity2d(40, iterations=1000)
    case, keep = X.make_case(model, config, pref)
    U, p = cases.fields(model)
    out = O.run(O.from_mesh2(mesh), case, 1000, U, p)
    assert np.isnan(out["R_uy"][0])
    d = out["done"]
    assert 100 < d < 1000
    assert out["R_ux"][d - 1] <= 1e-7 and out["R_p"][d - 1] <= 1e-7
    assert np.all(out["R_ux"][d:] == 1.0)
    assert out["U"][0].max() > 0.5 and out["U"][0].min() < -0.1


def test_golden_regression():
    g = np.load(os.path.join(GOLDEN, "cavity16_simple.npz"))
    mesh, model, config, pref = cases.cavity2d(16, iterations=int(g["iterations"]))
    case, keep = X.make_case(model, config, pref)
    U, p = cases.fields(model)
    out = O.run(O.from_mesh2(mesh), case, int(g["iterations"]), U, p)
    for k in ("R_ux", "R_p"):
        assert np.array_equal(out[k], g[k])
    assert np.array_equal(out["U"], g["U"]) and np.array_equal(out["p"], g["p"])


def _laplace_csr(nx, ny, shift=0.0, skew=0.0):
    """5-point operator on an nx x ny grid (rows in natural order), optionally
    with a diagonal shift and an antisymmetric convection-like skew."""
    n = nx * ny
    rows = []
    for j in range(ny):
        for i in range(nx):
            r = j * nx + i
            ent = {r: 4.0 + shift}
            for di, dj, sgn in ((-1, 0, 1), (1, 0, -1), (0, -1, 1), (0, 1, -1)):
                ii, jj = i + di, j + dj
                if 0 <= ii < nx and 0 <= jj < ny:
                    ent[jj * nx + ii] = -1.0 + sgn * skew
            rows.append(sorted(ent.items()))
    rp = np.zeros(n + 1, dtype=np.int32)
    col, val = [], []
    for r, ent in enumerate(rows):
        for c, v in ent:
            col.append(c)
            val.append(v)
        rp[r + 1] = len(col)
    return rp, np.array(col, dtype=np.int32), np.array(val)


def test_ilu0_matches_independent_ikj():
    """The oracle's ILU(0) equals a direct dense IKJ ILU(0) restricted to the
    pattern (Saad, Iterative Methods, Alg. 10.4) with the same operation order."""
    rp, col, val = _laplace_csr(5, 4, shift=0.3, skew=0.2)
    n = len(rp) - 1
    pat = {(r, int(col[q])) for r in range(n) for q in range(rp[r], rp[r + 1])}
    F = np.zeros((n, n))
    for r in range(n):
        for q in range(rp[r], rp[r + 1]):
            F[r, col[q]] = val[q]
    for i in range(n):
        for k in range(i):
            if (i, k) not in pat:
                continue
            F[i, k] = F[i, k] * (1.0 / F[k, k])
            for j in range(k + 1, n):
                if (i, j) in pat and (k, j) in pat:
                    F[i, j] = F[i, j] - F[i, k] * F[k, j]
    b = np.random.default_rng(3).standard_normal(n)
    y = np.zeros(n)
    for i in range(n):
        v = b[i]
        for k in range(i):
            if (i, k) in pat:
                v = v - F[i, k] * y[k]
        y[i] = v
    x = np.zeros(n)
    for i in range(n - 1, -1, -1):
        v = y[i]
        for j in range(n - 1, i, -1):
            if (i, j) in pat:
                v = v - F[i, j] * x[j]
        x[i] = v / F[i, i]
    assert np.array_equal(O.precon_apply(_abi.PRECON_ILU0, rp, col, val, b), x)


def test_ilu0_exact_on_tridiagonal_and_gmres_one_step():
    """ILU(0) of a tridiagonal matrix has no dropped fill, so it is the exact LU:
    M^{-1} A = I and preconditioned GMRES converges in one iteration."""
    rp, col, val = _laplace_csr(12, 1, shift=0.5, skew=0.3)
    n = len(rp) - 1
    A = np.zeros((n, n))
    for r in range(n):
        A[r, col[rp[r]:rp[r + 1]]] = val[rp[r]:rp[r + 1]]
    b = np.arange(1.0, n + 1)
    y = O.precon_apply(_abi.PRECON_ILU0, rp, col, val, b)
    assert np.allclose(A @ y, b, rtol=0, atol=1e-12)
    x, it, rn = O.linear_solve(_abi.SOLVER_GMRES, _abi.PRECON_ILU0, rp, col, val, b, np.zeros(n),
                               itmax=20, rtol=1e-12)
    assert it == 1 and np.allclose(A @ x, b, rtol=0, atol=1e-10)


@pytest.mark.parametrize("precon", [_abi.PRECON_NONE, _abi.PRECON_JACOBI, _abi.PRECON_DILU, _abi.PRECON_ILU0])
def test_gmres_solves_nonsymmetric_system(precon):
    """Full GMRES (no restart) on a nonsymmetric 2D convection-diffusion
    operator: converges within n iterations to the direct solution, with
    warm start, and reports iterations <= itmax."""
    rp, col, val = _laplace_csr(7, 6, shift=0.1, skew=0.35)
    n = len(rp) - 1
    A = np.zeros((n, n))
    for r in range(n):
        A[r, col[rp[r]:rp[r + 1]]] = val[rp[r]:rp[r + 1]]
    rng = np.random.default_rng(5)
    b = rng.standard_normal(n)
    x0 = 0.1 * rng.standard_normal(n)
    x, it, rn = O.linear_solve(_abi.SOLVER_GMRES, precon, rp, col, val, b, x0, itmax=n, atol=1e-13,
                               rtol=1e-13)
    xd = np.linalg.solve(A, b)
    assert 1 <= it <= n
    assert np.linalg.norm(x - xd) <= 1e-9 * np.linalg.norm(xd)
    # itmax caps the basis: 3 iterations, residual reported > tolerance
    x3, it3, rn3 = O.linear_solve(_abi.SOLVER_GMRES, precon, rp, col, val, b, x0, itmax=3, atol=1e-13,
                                  rtol=1e-13)
    assert it3 == 3 and rn3 > 1e-13
