"""Regenerates tests/golden/*.npz from the CPU oracle (run from the repo root):

    python tests/golden/make_golden.py

The vectors pin the oracle against accidental changes; they are the oracle's
own output (the reference's Julia run is not available to pin against)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "xcalibre_tw.jl_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402
import xcal as X  # noqa: E402
from xcal import cases  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

if __name__ == "__main__":
    its = 40
    mesh, model, config, pref = cases.cavity2d(16, iterations=its)
    case, keep = X.make_case(model, config, pref)
    U, p = cases.fields(model)
    out = O.run(O.from_mesh2(mesh), case, its, U, p)
    np.savez(os.path.join(HERE, "cavity16_simple.npz"), iterations=its, R_ux=out["R_ux"],
             R_uy=out["R_uy"], R_p=out["R_p"], U=out["U"], p=out["p"], krylov=out["krylov"])
    print("wrote cavity16_simple.npz", out["R_p"][-1])
