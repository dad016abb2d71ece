"""Shared helpers for the parity tests: run a case on the device (libxcal.so)
and on the CPU oracle with the same mesh numbering, and compare."""
import numpy as np

import oracle as O
import xcal as X
from xcal import _abi, cases

TOL = 1e-10   # FP64 device vs oracle: relative L2 bound on every field and history


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    fin = np.isfinite(a) & np.isfinite(b)
    if not np.array_equal(np.isfinite(a), np.isfinite(b)):
        return np.inf
    den = np.linalg.norm(b[fin])
    num = np.linalg.norm(a[fin] - b[fin])
    return num / den if den > 0 else num


def run_device(mesh, model, config, pref, iterations, renumber, piso=False, precision=_abi.PREC_FP64,
               tolerance=None, equations=True):
    """Run on the device; with equations=False only the residual histories,
    Krylov counts and fields come back (no mesh export or assembled systems)."""
    case, keep = X.make_case(model, config, pref, precision)
    s = X.Solver(mesh, renumber=renumber)
    try:
        s.setup(case)
        if tolerance is not None:
            s.set_tolerance(tolerance)
        U, p = cases.fields(model)
        s.set_field(_abi.FIELD_UX, U[0]); s.set_field(_abi.FIELD_UY, U[1]); s.set_field(_abi.FIELD_UZ, U[2])
        s.set_field(_abi.FIELD_P, p)
        if X.isturbulent(model):
            t = model.turbulence
            s.set_field(_abi.FIELD_K, t.k.values); s.set_field(_abi.FIELD_OMEGA, t.omega.values)
            s.set_field(_abi.FIELD_NUT, t.nut.values)
        out = s.run(iterations, piso=piso)
        if X.isturbulent(model):
            out["k"] = s.get_field(_abi.FIELD_K); out["omega"] = s.get_field(_abi.FIELD_OMEGA)
            out["nut"] = s.get_field(_abi.FIELD_NUT)
        out["U"] = np.stack([s.get_field(_abi.FIELD_UX), s.get_field(_abi.FIELD_UY), s.get_field(_abi.FIELD_UZ)])
        out["p"] = s.get_field(_abi.FIELD_P)
        out["ms"] = s.last_ms()
        if equations:
            out["perm"] = s.permutation() - 1
            out["dev_mesh"] = s.exported_mesh() if renumber != _abi.RENUMBER_NONE else mesh
            out["AU"], out["bU"] = s.equation(0)
            out["Ap"], bp = s.equation(1)
            out["bp"] = bp[0]
    finally:
        s.close()
    return out


def run_oracle(dev_mesh, model, config, pref, iterations, perm, piso=False):
    """Oracle on the device numbering; fields returned in the caller's numbering."""
    case, keep = X.make_case(model, config, pref)
    U, p = cases.fields(model)
    n = len(p)
    Ud = np.zeros_like(U)
    pd = np.zeros_like(p)
    Ud[:, perm] = U
    pd[perm] = p
    om = O.from_mesh2(dev_mesh)
    extra = {}
    if X.isturbulent(model):
        t = model.turbulence
        for name, f in (("k", t.k.values), ("omega", t.omega.values), ("nut", t.nut.values)):
            v = np.zeros_like(p)
            v[perm] = f
            extra[name] = v
    out = O.run(om, case, iterations, Ud, pd, piso=piso, ref_cell=int(perm[0]), want_eqns=True, **extra)
    out["U"] = out["U"][:, perm]
    out["p"] = out["p"][perm]
    for name in extra:
        out[name] = out[name][perm]
    return out


def compare(dev, orc, nU=2, check_eqns=True):
    """Return a dict of relative L2 differences (0.0 means bitwise equal)."""
    r = {}
    for k in ("R_ux", "R_uy", "R_p") + (("R_uz",) if nU == 3 else ()):
        r[k] = rel_l2(dev[k], orc[k])
    for d in range(nU):
        r[f"U{d}"] = rel_l2(dev["U"][d], orc["U"][d])
    r["p"] = rel_l2(dev["p"], orc["p"])
    for name in ("k", "omega", "nut"):
        if name in dev:
            r[name] = rel_l2(dev[name], orc[name])
    if check_eqns:
        r["AU"] = rel_l2(dev["AU"], orc["AU"])
        r["Ap"] = rel_l2(dev["Ap"], orc["Ap"])
        r["bp"] = rel_l2(dev["bp"], orc["bp"])
        for d in range(nU):
            r[f"bU{d}"] = rel_l2(dev["bU"][d], orc["bU"][d])
    return r


def assert_parity(dev, orc, nU=2, tol=TOL, check_eqns=True):
    assert dev["done"] == orc["done"], (dev["done"], orc["done"])
    k_dev = dev["krylov"][: dev["done"]]
    k_orc = orc["krylov"][: orc["done"]]
    cols = [0, 1, 3] + ([2] if nU == 3 else [])
    assert np.array_equal(k_dev[:, cols], k_orc[:, cols]), "Krylov iteration counts differ"
    diffs = compare(dev, orc, nU, check_eqns)
    bad = {k: v for k, v in diffs.items() if not v <= tol}
    assert not bad, f"relative L2 above {tol}: {bad}"
    return diffs
