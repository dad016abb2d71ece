"""The 128^3 lid-driven cavity (2,097,152 hexahedra, the 3D benchmark size) is
too large for the CPU oracle, so it is checked through properties that hold at
any size, after two SIMPLE iterations on the device (FP64):

* the assembled pressure matrix (Laplacian(rDf, p) + setReference!) is exactly
  symmetric, as its face coefficients are shared by both cells;
* its rows sum to zero up to rounding, except the reference cell's row (all
  walls are Neumann for p), which setReference! doubled;
* residual! recomputed on the assembled system with the standalone operator
  (xcal_residual) reproduces the run's R_p of the last iteration bit for bit;
* residuals and fields are finite (except R_uy, R_uz of the first iteration,
  0/0 as in the reference) and the Krylov counts are within itmax.
"""

import numpy as np
import pytest

import xcal as X
from xcal import _abi, cases

pytestmark = pytest.mark.gpu


def test_cavity128_properties():
    its = 2
    mesh, model, config, pref = cases.cavity3d(128, iterations=its)
    case, keep = X.make_case(model, config, pref)
    s = X.Solver(mesh, renumber=_abi.RENUMBER_COLOR)
    try:
        s.setup(case)
        U0, p0 = cases.fields(model)
        for f, v in ((_abi.FIELD_UX, U0[0]), (_abi.FIELD_UY, U0[1]), (_abi.FIELD_UZ, U0[2]), (_abi.FIELD_P, p0)):
            s.set_field(f, v)
        out = s.run(its)
        p_user = s.get_field(_abi.FIELD_P)
        U = [s.get_field(f) for f in (_abi.FIELD_UX, _abi.FIELD_UY, _abi.FIELD_UZ)]
        perm = s.permutation() - 1
        rp, col, fl, bl, nl = s.csr()
        Ap, bp = s.equation(1)
        ref_dev = int(perm[0])
        lib = _abi.load()
        n = mesh.ncells
        p_dev = np.empty(n)
        p_dev[perm] = p_user
        R = np.zeros(1)
        _abi.check(lib.xcal_residual(s.ctx, n, _abi.i32ptr(rp), _abi.i32ptr(col), _abi.dptr(Ap),
                                     _abi.dptr(p_dev), _abi.dptr(bp[0]), _abi.dptr(R)), s.ctx, "xcal_residual")
    finally:
        s.close()
    assert out["done"] == its
    kr = out["krylov"][:its]
    assert np.all(kr[:, :4] <= 100)
    # R_uy and R_uz of the first iteration are 0/0 in the reference as well
    # (their right-hand sides are exactly zero when the lid moves along x)
    for k in ("R_ux", "R_p"):
        assert np.all(np.isfinite(out[k][:its])), k
    for k in ("R_uy", "R_uz"):
        assert np.isnan(out[k][0]) and np.all(np.isfinite(out[k][1:its])), k
    assert np.all(np.isfinite(p_user)) and all(np.all(np.isfinite(u)) for u in U)
    # symmetry: entry (i, j) equals entry (j, i), bitwise
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp))
    c64 = col.astype(np.int64)
    key = rows * n + c64
    tkey = c64 * n + rows
    order = np.argsort(key)
    pos = np.searchsorted(key[order], tkey)
    assert np.array_equal(key[order][pos], tkey), "pattern not symmetric"
    assert np.array_equal(Ap, Ap[order][pos]), "pressure matrix not symmetric"
    # zero row sums away from the reference cell
    rs = np.add.reduceat(Ap, rp[:-1].astype(np.int64))
    scale = np.abs(Ap).max()
    mask = np.ones(n, dtype=bool)
    mask[ref_dev] = False
    assert np.abs(rs[mask]).max() <= 1e-12 * scale
    diag = Ap[np.flatnonzero(c64 == rows)]
    assert rs[ref_dev] == pytest.approx(diag[ref_dev] / 2.0, rel=1e-12)
    # residual! on the assembled system equals the run's R_p
    assert R[0] == out["R_p"][its - 1]
