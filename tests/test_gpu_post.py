"""Post-processing on a context's device fields: wall_shear_stress,
pressure_force, viscous_force (src/Postprocess/Postprocess_forces.jl:5-94,
surface_normal_gradient in src/Calculate/Calculate_5_surface_normal_gradient.jl:20-37)
and model2vtk, checked against a numpy restatement of the reference formulas
on the fields read back from the device."""
import numpy as np
import pytest

import xcal as X
from xcal import _abi, cases

pytestmark = pytest.mark.gpu


def _restate(mesh, U, p, nut, nu, patch, Uw, rho):
    pid = mesh.boundary_index(patch) - 1
    a, b = mesh.patch_ptr[pid], mesh.patch_ptr[pid + 1]
    fn = mesh.face_normal.reshape(-1, 3)
    fc = mesh.face_centre.reshape(-1, 3)
    tau, pos = [], []
    Fp = np.zeros(3)
    Fv = np.zeros(3)
    for k in range(a, b):
        f, c = mesh.patch_faces[k] - 1, mesh.patch_cells[k] - 1
        n = fn[f]
        ud = U[:, c] - Uw
        dn = (ud[0] * n[0] + ud[1] * n[1]) + ud[2] * n[2]
        g = (ud - dn * n) / mesh.face_delta[f]
        tau.append(g * (nu + nut[c]))
        pos.append(fc[f])
        for d in range(3):
            Fp[d] += p[c] * (mesh.face_area[f] * n[d])
            Fv[d] += g[d] * mesh.face_area[f] * (nu + nut[c])
    return np.array(tau), np.array(pos), rho * Fp, rho * Fv


@pytest.mark.parametrize("which", ["cavity", "flatplate"])
def test_wall_shear_and_forces(which, tmp_path):
    if which == "cavity":
        mesh, model, config, pref = cases.cavity2d(16, iterations=40)
        patch, Uw, its = "top", np.array([1.0, 0.0, 0.0]), 40
    else:
        mesh, model, config, pref = cases.flatplate(40, 20, iterations=30)
        patch, Uw, its = "wall", np.zeros(3), 30
    case, keep = X.make_case(model, config, pref)
    s = X.Solver(mesh, renumber=_abi.RENUMBER_COLOR)
    try:
        s.setup(case)
        Uf, pf = cases.fields(model)
        for f, v in ((_abi.FIELD_UX, Uf[0]), (_abi.FIELD_UY, Uf[1]), (_abi.FIELD_UZ, Uf[2]), (_abi.FIELD_P, pf)):
            s.set_field(f, v)
        if X.isturbulent(model):
            t = model.turbulence
            s.set_field(_abi.FIELD_K, t.k.values); s.set_field(_abi.FIELD_OMEGA, t.omega.values)
            s.set_field(_abi.FIELD_NUT, t.nut.values)
        s.run(its, want_krylov=False)
        U = np.stack([s.get_field(_abi.FIELD_UX), s.get_field(_abi.FIELD_UY), s.get_field(_abi.FIELD_UZ)])
        p = s.get_field(_abi.FIELD_P)
        nut = s.get_field(_abi.FIELD_NUT) if X.isturbulent(model) else np.zeros(mesh.ncells)
        tau, pos = s.wall_shear_stress(patch)
        Fp = s.pressure_force(patch, 1.2)
        Fv = s.viscous_force(patch, 1.2)
        s.model2vtk(str(tmp_path / "m"))
    finally:
        s.close()
    t_ref, p_ref, Fp_ref, Fv_ref = _restate(mesh, U, p, nut, model.nu.values, patch, Uw, 1.2)
    assert np.array_equal(tau, t_ref) and np.array_equal(pos, p_ref)
    assert np.array_equal(Fp, Fp_ref) and np.array_equal(Fv, Fv_ref)
    assert np.abs(tau).max() > 0.0
    text = open(str(tmp_path / "m") + ".vtk").read().split("\n")
    k = text.index("SCALARS p double 1")
    assert np.array_equal(np.array([float(x) for x in text[k + 2:k + 2 + mesh.ncells]]), p)
    if X.isturbulent(model):
        k = text.index("SCALARS nut double 1")
        assert np.array_equal(np.array([float(x) for x in text[k + 2:k + 2 + mesh.ncells]]), nut)
