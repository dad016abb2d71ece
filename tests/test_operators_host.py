"""Operator-level API without a GPU: the Python operator algebra (signs,
schemes, model building as ModelFramework_1_operations.jl:3-58 defines them)
and the oracle's generic assembly against structural invariants and a known
answer."""
import numpy as np

import oracle as O
import xcal as X
from xcal import _abi, cases, meshgen
from xcal import operators as op


def test_operator_algebra_signs():
    mesh = X.build_mesh(cases._unv("cavity", meshgen.cavity_unv, n=4, L=0.1))
    phi = X.ScalarField(mesh)
    f = np.ones(mesh.nfaces)
    m = (op.Time(phi) + op.Laplacian(f, phi) - op.Divergence[op.Upwind](f, phi) == -op.Source(np.ones(16)))
    assert [t.sign for t in m.terms] == [1.0, 1.0, -1.0]
    assert [s.sign for s in m.sources] == [-1.0]
    assert m.terms[2].scheme is op.Upwind and m.terms[0].scheme is op.Steady


def test_oracle_generic_assembly_invariants_and_known_answer():
    """Laplacian(1, phi) == Source(0) on a uniform cavity with phi = 1 on the
    left (inlet) and 0 on the right (outlet): interior rows sum to zero, the
    pattern is symmetric in value, and the discrete solution is linear in x
    (exact for orthogonal uniform meshes)."""
    mesh = O.build_unv(cases._unv("cavity", meshgen.cavity_unv, n=10, L=0.1)).to_mesh2()
    om = O.from_mesh2(mesh)
    n = mesh.ncells
    terms = (_abi.Term * 1)()
    f = np.ones(mesh.nfaces)
    terms[0].kind, terms[0].scheme, terms[0].sign = _abi.TERM_LAPLACIAN, 0, 1.0
    terms[0].flux = _abi.dptr(f)
    srcs = (_abi.Source * 1)()
    z = np.zeros(n)
    srcs[0].sign, srcs[0].field = 1.0, _abi.dptr(z)
    bcs = (_abi.BC * 4)()
    for k, (name, t, v) in enumerate((("inlet", _abi.BC_DIRICHLET, 1.0), ("outlet", _abi.BC_DIRICHLET, 0.0),
                                      ("bottom", _abi.BC_NEUMANN, 0.0), ("top", _abi.BC_NEUMANN, 0.0))):
        bcs[k].patch, bcs[k].type = mesh.boundary_index(name) - 1, t
        bcs[k].value[:] = (v, v, v)
    A0, b0 = O.assemble(om, terms, 1, srcs, 1, bcs, 0)
    rp, col = om.pattern()
    rows = np.repeat(np.arange(n), np.diff(rp))
    assert np.allclose(np.bincount(rows, weights=A0, minlength=n), 0.0, atol=1e-15)
    At = {(r, c): v for r, c, v in zip(rows, col, A0)}
    assert all(At[(r, c)] == At[(c, r)] for (r, c) in At)
    A, b = O.assemble(om, terms, 1, srcs, 1, bcs, 4)
    x, its, rn = O.linear_solve(_abi.SOLVER_CG, _abi.PRECON_DILU, rp, col, A, b, np.zeros(n), itmax=500,
                                atol=1e-14, rtol=1e-14)
    xc = mesh.cell_centre.reshape(n, 3)[:, 0]
    assert np.allclose(x, 1.0 - xc / 0.1, atol=1e-10)
