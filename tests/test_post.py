"""VTK writer (write_vtk / model2vtk, src/VTK/VTK_writer.jl:3-116) through the
C ABI (xcal_vtk_write runs on the host, no GPU needed): structure as the
reference writes it, and every number parses back to the exact double."""
import os

import numpy as np
import pytest

import xcal as X
from xcal import cases, meshgen


def _parse(path):
    lines = open(path).read().split("\n")
    assert lines[:4] == ["# vtk DataFile Version 3.0", "jCFD simulation data", "ASCII",
                         "DATASET UNSTRUCTURED_GRID"]
    return lines


def _check(path, mesh, fields):
    L = _parse(path)
    i = 4
    assert L[i] == f"POINTS {mesh.nnodes} double"
    pts = np.array([[float(t) for t in L[i + 1 + k].split(" ")] for k in range(mesh.nnodes)])
    assert np.array_equal(pts.ravel(), mesh.node_coords)
    i += 1 + mesh.nnodes
    cnp = mesh.cell_nodes_ptr - 1
    tot = int(cnp[-1])
    assert L[i] == f"CELLS {mesh.ncells} {tot + mesh.ncells}"
    for c in range(mesh.ncells):
        ids = mesh.cell_nodes[cnp[c]:cnp[c + 1]] - 1
        # println(io, nNodes, " ", nodes) with nodes = " id0 id1 ...": two spaces after the count
        assert L[i + 1 + c] == f"{len(ids)}  " + " ".join(str(int(x)) for x in ids)
    i += 1 + mesh.ncells
    assert L[i] == f"CELL_TYPES {mesh.ncells}"
    for c in range(mesh.ncells):
        k = cnp[c + 1] - cnp[c]
        assert L[i + 1 + c] == {3: "5", 4: "9"}.get(k, "7")
    i += 1 + mesh.ncells
    assert L[i] == f"CELL_DATA {mesh.ncells}"
    i += 1
    for label, kind, vals in fields:
        if kind == 1:
            assert L[i] == f"SCALARS {label} double 1" and L[i + 1] == "LOOKUP_TABLE CellColors"
            got = np.array([float(t) for t in L[i + 2:i + 2 + mesh.ncells]])
            assert np.array_equal(got, vals)
            i += 2 + mesh.ncells
        else:
            assert L[i] == f"VECTORS {label} double"
            got = np.array([[float(t) for t in L[i + 1 + c].split(" ")] for c in range(mesh.ncells)])
            assert np.array_equal(got.T, vals)
            i += 1 + mesh.ncells
    assert L[i:] == [""]


def test_write_vtk_cavity(tmp_path):
    mesh, model, config, pref = cases.cavity2d(7, iterations=1)
    rng = np.random.default_rng(1)
    n = mesh.ncells
    model.U.x.values[:] = rng.standard_normal(n) * 1e-7
    model.U.y.values[:] = rng.standard_normal(n) * 1e6
    model.p.values[:] = rng.standard_normal(n)
    name = str(tmp_path / "cav")
    X.model2vtk(model, name)
    U = np.stack([model.U.x.values, model.U.y.values, model.U.z.values])
    _check(name + ".vtk", mesh, [("U", 3, U), ("p", 1, model.p.values)])


def test_write_vtk_reference_triangles(ref_meshes, tmp_path):
    mesh = X.build_mesh(os.path.join(ref_meshes, "trig40.unv"))
    f = X.ScalarField(mesh)
    f.values[:] = np.arange(mesh.ncells) / 7.0
    X.write_vtk(str(tmp_path / "trig"), mesh, ("phi", f))
    _check(str(tmp_path / "trig") + ".vtk", mesh, [("phi", 1, f.values)])


def test_write_vtk_needs_nodes_and_valid_fields(tmp_path):
    m = meshgen.hex_cavity(3)
    mesh = X.Mesh2.from_dict(m)           # generated without node data
    f = X.ScalarField(mesh)
    with pytest.raises(X._abi.XcalError):
        X.write_vtk(str(tmp_path / "x"), mesh, ("phi", f))
    mesh2, model, config, pref = cases.cavity2d(4, iterations=1)
    with pytest.raises(TypeError):
        X.write_vtk(str(tmp_path / "y"), mesh2, ("phi", np.zeros(16)))
