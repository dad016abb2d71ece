"""Host side of libxcal.so without a GPU: the C ABI loads and exports every
symbol of include/xcal.h; the UNV builder, renumbering, CSR pattern and DILU
level sets are bit-exact against the oracle's independent implementations."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle as O
import xcal as X
from xcal import _abi, cases, meshgen
from xcal.mesh import ARRAY_FIELDS, Mesh2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "xcal.h")).read()
    return sorted(set(re.findall(r"^int\s+(xcal_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_header_symbol():
    lib = _abi.load()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
        assert s in _abi.SIGNATURES, f"{s} missing from the ctypes mirror"
    major, minor = C.c_int32(), C.c_int32()
    assert lib.xcal_version(C.byref(major), C.byref(minor)) == 0


def test_ctx_create_without_device_fails_cleanly():
    if os.environ.get("CUDA_VISIBLE_DEVICES", None) is None and _has_gpu():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert _abi.load().xcal_ctx_create(0, 0, C.byref(h)) == -4   # XCAL_ERR_CUDA


def test_serve_config_validation():
    """xcal_serve_create checks its configuration before touching a device."""
    lib = _abi.load()
    h = C.c_void_p()
    for bad in (dict(slots=0), dict(slots=5000), dict(max_iterations=0), dict(tolerance=-1.0),
                dict(renumber=7), dict(precision=3), dict(dim=1), dict(max_ctas=-1), dict(device_bytes=-1.0)):
        cfg = dict(slots=2, max_iterations=10, renumber=2, precision=1, tolerance=1e-6, dim=2)
        cfg.update(bad)
        assert lib.xcal_serve_create(0, C.byref(_abi.ServeCfg(**cfg)), C.byref(h)) == -1, bad
    assert lib.xcal_serve_poll(None, 1, 0, None, None, None) == -1
    assert lib.xcal_ctx_set_tolerance(None, 1e-6) == -1


def test_package_import_leaves_the_environment_alone():
    """Importing the package changes no process-wide setting (the serving
    loop needs no driver configuration: it runs as one launch)."""
    import subprocess
    import sys
    pkg = os.path.join(os.path.dirname(__file__), "..", "xcalibre_tw.jl_b200")
    code = ("import os, sys; before = dict(os.environ); sys.path.insert(0, sys.argv[1]); import xcal; "
            "print(dict(os.environ) == before)")
    out = subprocess.run([sys.executable, "-c", code, pkg], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "True"


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def _same(a, b):
    return [k for k, _ in ARRAY_FIELDS if not np.array_equal(getattr(a, k), getattr(b, k))]


@pytest.mark.parametrize("name", ["quad40.unv", "trig40.unv", "quad.unv", "backwardFacingStep_10mm.unv"])
def test_builder_matches_oracle_on_reference_meshes(ref_meshes, name):
    path = os.path.join(ref_meshes, name)
    a = X.build_mesh(path, scale=0.001)
    b = O.build_unv(path, scale=0.001).to_mesh2()
    assert _same(a, b) == []
    assert a.patch_names == b.patch_names


def test_builder_matches_oracle_on_generated_meshes():
    for fn, kw in ((meshgen.cavity_unv, dict(n=20, L=0.1)), (meshgen.bfs_unv, dict(cells_per_h=9)),
                   (meshgen.flatplate_unv, dict(nx=40, ny=30))):
        path = f"/tmp/xcal_host_{fn.__name__}.unv"
        fn(path, **kw)
        assert _same(X.build_mesh(path), O.build_unv(path).to_mesh2()) == []


def test_builder_rejects_bad_input(tmp_path):
    with pytest.raises(_abi.XcalError):
        X.build_mesh(str(tmp_path / "missing.unv"))
    bad = tmp_path / "bad.unv"
    bad.write_text("    -1\n  2412\n         1        11         2         1         7         2\n"
                   "         0         1         1\n         5         5\n    -1\n")
    with pytest.raises(_abi.XcalError):
        X.build_mesh(str(bad))


def _hmesh(mesh):
    lib = _abi.load()
    h = C.c_void_p()
    err = C.create_string_buffer(256)
    st = lib.xcal_hmesh_from_desc(C.byref(mesh.desc()), C.byref(h), err, 256)
    assert st == 0, err.value
    return h


def _renumber(mesh, mode):
    lib = _abi.load()
    h = _hmesh(mesh)
    out = C.c_void_p()
    perm = np.zeros(mesh.ncells, dtype=np.int64)
    assert lib.xcal_hmesh_renumber(h, mode, C.byref(out), _abi.i64ptr(perm)) == 0
    d = _abi.MeshDesc()
    lib.xcal_hmesh_desc(out, C.byref(d))
    m2 = Mesh2.from_desc(d, mesh.patch_names)
    n = mesh.ncells
    cap = n + len(mesh.cell_faces)
    nnz = np.zeros(1, dtype=np.int64)
    rp = np.zeros(n + 1, dtype=np.int32)
    col = np.zeros(cap, dtype=np.int32)
    fl = np.zeros(n, dtype=np.int32)
    bl = np.zeros(n, dtype=np.int32)
    nl = np.zeros(2, dtype=np.int32)
    assert lib.xcal_hmesh_csr(out, _abi.i64ptr(nnz), _abi.i32ptr(rp), _abi.i32ptr(col), _abi.i32ptr(fl),
                              _abi.i32ptr(bl), _abi.i32ptr(nl)) == 0
    lib.xcal_hmesh_free(out)
    lib.xcal_hmesh_free(h)
    return perm - 1, m2, rp, col[: int(nnz[0])], fl, bl, nl


@pytest.mark.parametrize("mode", [_abi.RENUMBER_NONE, _abi.RENUMBER_RCM, _abi.RENUMBER_COLOR])
def test_renumbering_csr_levels_match_oracle(mode):
    path = cases._unv("bfs", meshgen.bfs_unv, cells_per_h=9)
    mesh = X.build_mesh(path)
    perm, m2, rp, col, fl, bl, nl = _renumber(mesh, mode)
    om = O.from_mesh2(mesh)
    assert np.array_equal(perm, om.renumber(mode))            # bit-exact permutation
    # the renumbered mesh is a valid reference-layout mesh with the same geometry
    assert np.array_equal(np.sort(m2.cell_volume), np.sort(mesh.cell_volume))
    assert np.array_equal(m2.cell_volume[perm], mesh.cell_volume)
    o2 = O.from_mesh2(m2)
    colptr, rowval = o2.pattern()                             # Equation(mesh) pattern
    assert np.array_equal(rp, colptr) and np.array_equal(col, rowval)
    ofl, obl = O.levels(rp, col)
    assert np.array_equal(fl, ofl) and np.array_equal(bl, obl)
    if mode == _abi.RENUMBER_COLOR:
        assert tuple(nl) == (2, 2)                             # quad mesh: two colours
    if mode == _abi.RENUMBER_NONE:
        assert _same(m2, mesh) == []


def test_mesh_from_desc_validation():
    path = cases._unv("cavity", meshgen.cavity_unv, n=8, L=0.1)
    mesh = X.build_mesh(path)
    bad = mesh.copy()
    bad.cell_neighbours[0] = mesh.ncells + 5
    lib = _abi.load()
    h = C.c_void_p()
    err = C.create_string_buffer(256)
    assert lib.xcal_hmesh_from_desc(C.byref(bad.desc()), C.byref(h), err, 256) == -2
    assert b"out of range" in err.value
    bad = mesh.copy()
    bad.cell_volume[3] = -1.0
    assert lib.xcal_hmesh_from_desc(C.byref(bad.desc()), C.byref(h), err, 256) == -2


def test_api_errors_like_reference():
    path = cases._unv("cavity", meshgen.cavity_unv, n=8, L=0.1)
    mesh = X.build_mesh(path)
    model = X.RANS(X.Laminar, mesh=mesh, viscosity=X.ConstantScalar(1e-3))
    with pytest.raises(KeyError):
        X.assign(model, "U", X.Dirichlet("nowhere", [0, 0, 0]))
    with pytest.raises(ValueError):
        X.Dirichlet("inlet", [1, 2])
    with pytest.raises(ValueError):
        X.initialise(model.U, [1, 2])
    X.assign(model, "U", X.Dirichlet("inlet", [0, 0, 0]))
    X.assign(model, "p", X.Neumann("inlet", 0.0))
    solvers = dict(U=X.set_solver(model.U, solver=X.GmresSolver, preconditioner=X.DILU(),
                                  convergence=1e-7, relax=0.7),
                   p=X.set_solver(model.p, solver=X.CgSolver, preconditioner=X.LDL(),
                                  convergence=1e-7, relax=0.3))
    cfg = X.Configuration(solvers=solvers, schemes=dict(U=X.set_schemes(), p=X.set_schemes()),
                          runtime=X.set_runtime(10))
    with pytest.raises(_abi.XcalError):
        X.make_case(model, cfg)
