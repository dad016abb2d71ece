"""Copies the reference project's own test fixtures used by the tests into
this folder (run from the repo root where the reference is mounted):

    python tests/golden/reference/copy_fixtures.py /path/to/reference

* unv_sample_meshes/{quad40,trig40,quad,backwardFacingStep_10mm}.unv, gzip-
  compressed: the reference's sample meshes that pin the UNV reader, the mesh
  builder's numbering and the VTK writer (quad40: 1600 cells, 3280 faces, 160
  boundary faces);
* flatplate_OF_wall_laminar.csv reduced to the columns the laminar flat-plate
  skin-friction check reads (arc_length, wallShearStress:0, wallShearStress:1),
  the OpenFOAM wall data the reference compares its own laminar flat plate with
  (CASE_UNV_flatplate.jl:67-83: U = 0.2 m/s, nu = 1e-5).

The files are data, copied unchanged apart from the compression and the column
selection; the tests read them from here, so they run without the reference."""
import gzip
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MESHES = ("quad40.unv", "trig40.unv", "quad.unv", "backwardFacingStep_10mm.unv")

if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("XCAL_REFERENCE_ROOT", "")
    if not os.path.isdir(ref):
        raise SystemExit("usage: copy_fixtures.py <reference project root>")
    for name in MESHES:
        with open(os.path.join(ref, "unv_sample_meshes", name), "rb") as src, \
                gzip.open(os.path.join(HERE, name + ".gz"), "wb", compresslevel=9) as dst:
            shutil.copyfileobj(src, dst)
    data = np.loadtxt(os.path.join(ref, "flatplate_OF_wall_laminar.csv"), delimiter=",", skiprows=1)
    np.savez_compressed(os.path.join(HERE, "flatplate_OF_wall_laminar.npz"), arc_length=data[:, 6],
                        tau_x=data[:, 8], tau_y=data[:, 9])
    print("copied", MESHES, "and the laminar flat-plate wall data")
