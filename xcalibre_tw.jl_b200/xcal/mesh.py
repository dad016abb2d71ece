"""Host-side mesh container in the reference's flattened layout.

Mirrors ``Mesh.Mesh2`` after ``update_mesh_format``
(src/Mesh/Mesh_0_types.jl:82-94, src/Mesh/Mesh2D/Mesh2D_0_update_mesh.jl:5-142):
1-based int64 connectivity, float64 geometry, boundary faces numbered first.
"""
import ctypes as C

import numpy as np

from . import _abi

ARRAY_FIELDS = (
    ("cell_centre", np.float64), ("cell_volume", np.float64),
    ("cell_faces_ptr", np.int64), ("cell_faces", np.int64), ("cell_neighbours", np.int64),
    ("cell_nsign", np.int64), ("face_owner", np.int64), ("face_centre", np.float64),
    ("face_normal", np.float64), ("face_e", np.float64), ("face_area", np.float64),
    ("face_delta", np.float64), ("face_weight", np.float64), ("patch_ptr", np.int64),
    ("patch_faces", np.int64), ("patch_cells", np.int64),
)


# optional node data (mesh.nodes, mesh.cell_nodes), used by the VTK writer
NODE_FIELDS = (("node_coords", np.float64), ("cell_nodes_ptr", np.int64), ("cell_nodes", np.int64))


class Mesh2:
    """Flattened mesh.  ``boundaries`` lists patch names in file order;
    ``boundary_index(name)`` is 1-based like the reference."""

    def __init__(self, ncells, nfaces, nbfaces, dim, patch_names, **arrays):
        self.ncells = int(ncells)
        self.nfaces = int(nfaces)
        self.nbfaces = int(nbfaces)
        self.dim = int(dim)
        self.patch_names = list(patch_names)
        for name, dt in ARRAY_FIELDS:
            setattr(self, name, np.ascontiguousarray(arrays[name], dtype=dt))
        for name, dt in NODE_FIELDS:
            setattr(self, name, np.ascontiguousarray(arrays.get(name, np.zeros(0)), dtype=dt))
        self.nnodes = len(self.node_coords) // 3
        self._desc = None

    # --- reference helpers (src/Mesh/Mesh_1_functions.jl)
    def total_boundary_faces(self):
        return int(self.patch_ptr[-1])

    def boundary_index(self, name):
        name = name.lstrip(":") if isinstance(name, str) else name
        for i, n in enumerate(self.patch_names):
            if n == name:
                return i + 1
        raise KeyError(f"boundary {name!r} not found; patches: {self.patch_names}")

    @property
    def boundaries(self):
        out = []
        for i, n in enumerate(self.patch_names):
            a, b = self.patch_ptr[i], self.patch_ptr[i + 1]
            out.append((n, self.patch_faces[a:b], self.patch_cells[a:b]))
        return out

    def cell_centres(self):
        return self.cell_centre.reshape(-1, 3)

    def desc(self):
        """ctypes MeshDesc pointing at this object's arrays (kept alive by self)."""
        d = _abi.MeshDesc()
        d.ncells, d.nfaces, d.nbfaces, d.dim = self.ncells, self.nfaces, self.nbfaces, self.dim
        for name, dt in ARRAY_FIELDS:
            arr = getattr(self, name)
            ptype = _abi.P_d if dt == np.float64 else _abi.P_i64
            setattr(d, name, arr.ctypes.data_as(ptype))
        d.npatches = len(self.patch_names)
        if self.nnodes > 0:
            d.nnodes = self.nnodes
            d.node_coords = self.node_coords.ctypes.data_as(_abi.P_d)
            d.cell_nodes_ptr = self.cell_nodes_ptr.ctypes.data_as(_abi.P_i64)
            d.cell_nodes = self.cell_nodes.ctypes.data_as(_abi.P_i64)
        self._desc = d
        return d

    @classmethod
    def from_desc(cls, d, patch_names):
        """Copy a MeshDesc (pointers owned elsewhere) into numpy arrays."""
        nc, nf = d.ncells, d.nfaces
        tot = None
        ptr = np.ctypeslib.as_array(d.cell_faces_ptr, shape=(nc + 1,)).copy()
        tot = int(ptr[-1] - 1)
        npch = d.npatches
        pptr = np.ctypeslib.as_array(d.patch_ptr, shape=(npch + 1,)).copy()
        plen = int(pptr[-1])
        shapes = {
            "cell_centre": 3 * nc, "cell_volume": nc, "cell_faces_ptr": nc + 1,
            "cell_faces": tot, "cell_neighbours": tot, "cell_nsign": tot,
            "face_owner": 2 * nf, "face_centre": 3 * nf, "face_normal": 3 * nf,
            "face_e": 3 * nf, "face_area": nf, "face_delta": nf, "face_weight": nf,
            "patch_ptr": npch + 1, "patch_faces": plen, "patch_cells": plen,
        }
        arrays = {}
        for name, dt in ARRAY_FIELDS:
            n = shapes[name]
            arrays[name] = np.ctypeslib.as_array(getattr(d, name), shape=(n,)).copy() if n else np.zeros(0, dt)
        if d.nnodes > 0 and d.cell_nodes_ptr:
            cnp = np.ctypeslib.as_array(d.cell_nodes_ptr, shape=(nc + 1,)).copy()
            arrays["node_coords"] = np.ctypeslib.as_array(d.node_coords, shape=(3 * d.nnodes,)).copy()
            arrays["cell_nodes_ptr"] = cnp
            arrays["cell_nodes"] = np.ctypeslib.as_array(d.cell_nodes, shape=(int(cnp[-1] - 1),)).copy()
        return cls(nc, nf, d.nbfaces, d.dim, patch_names, **arrays)

    @classmethod
    def from_dict(cls, m):
        arrays = {k: m[k] for k, _ in ARRAY_FIELDS}
        return cls(m["ncells"], m["nfaces"], m["nbfaces"], m["dim"], m["patch_names"], **arrays)

    def copy(self):
        return Mesh2(self.ncells, self.nfaces, self.nbfaces, self.dim, self.patch_names,
                     **{k: getattr(self, k).copy() for k, _ in ARRAY_FIELDS + NODE_FIELDS})
