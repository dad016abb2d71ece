"""How the cell numbering changes the reference's SIMPLE run -- TEST
INFRASTRUCTURE (oracle only, no product code):

    python oracle/numbering_report.py [--cases cavity,bfs] [--iterations 3000]

For each case and each numbering (none = the caller's, i.e. the reference's own
order; rcm; color = the device default), runs the CPU restatement to the 1e-7
stop of the reference and prints one JSON line: outer iterations to converge,
mean Krylov iterations per outer iteration (p CG, U BiCGSTAB), the DILU level
counts of the numbering (phases per preconditioner sweep on the device), and
the relative L2 difference of the converged fields from the reference-order
run's.  DILU depends on the row order, so the numberings converge along
different paths to the same discrete steady solution."""
import argparse
import json
import multiprocessing as mp
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "xcalibre_tw.jl_b200"))


def one(args):
    name, mode, its = args
    import numpy as np
    import oracle as O
    import xcal as X
    from xcal import cases, meshgen
    if name == "cavity":
        mesh = O.build_unv(cases._unv("cavity", meshgen.cavity_unv, n=40, L=0.1)).to_mesh2()
        mesh, model, config, pref = cases.cavity2d(40, iterations=its, mesh=mesh)
    else:
        mesh = O.build_unv(cases._unv("bfs", meshgen.bfs_unv, cells_per_h=27)).to_mesh2()
        mesh, model, config, pref = cases.bfs(27, iterations=its, mesh=mesh)
    dev_mesh, perm = O.renumbered(mesh, mode)
    om = O.from_mesh2(dev_mesh)
    rp, col = om.pattern()
    fl, bl = O.levels(rp, col)
    case, keep = X.make_case(model, config, pref)
    U, p = cases.fields(model)
    Ud, pd = np.zeros_like(U), np.zeros_like(p)
    Ud[:, perm] = U
    pd[perm] = p
    out = O.run(om, case, its, Ud, pd, ref_cell=int(perm[0]))
    done = out["done"]
    k = out["krylov"][:done]
    return dict(case=name, numbering=["none", "rcm", "color"][mode], outer_iterations=done,
                converged=bool(done < its), p_cg_mean=float(k[:, 3].mean()), U_bicgstab_mean=float(k[:, 0].mean()),
                p_cg_at_itmax_fraction=float((k[:, 3] >= 100).mean()),
                dilu_levels=[int(fl.max()) + 1, int(bl.max()) + 1], loop_seconds=out["loop_seconds"],
                U=out["U"][:, perm].tolist(), p=out["p"][perm].tolist())


if __name__ == "__main__":
    import numpy as np
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", default="cavity,bfs")
    ap.add_argument("--iterations", type=int, default=3000)
    a = ap.parse_args()
    jobs = [(c, m, a.iterations) for c in a.cases.split(",") for m in (0, 1, 2)]
    with mp.get_context("spawn").Pool(min(len(jobs), os.cpu_count() or 1)) as pool:
        res = pool.map(one, jobs)
    for c in a.cases.split(","):
        ref = [r for r in res if r["case"] == c and r["numbering"] == "none"][0]
        for r in [r for r in res if r["case"] == c]:
            rel = {}
            for nm, a_, b_ in (("Ux", r["U"][0], ref["U"][0]), ("Uy", r["U"][1], ref["U"][1]), ("p", r["p"], ref["p"])):
                a_, b_ = np.array(a_), np.array(b_)
                rel[nm] = float(np.linalg.norm(a_ - b_) / max(np.linalg.norm(b_), 1e-300))
            row = {k: v for k, v in r.items() if k not in ("U", "p")}
            row["rel_l2_vs_reference_order"] = rel
            print(json.dumps(row))
