"""Benchmark of the SIMPLE hot path on one B200 (per rank).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl xcal|reference]
                    [--config cavity3d|bfs|cavity|flatplate|serve] [--size S]
                    [--precision both|fp64|mixed] [--renumber color|rcm|none]

Default workload: the 3D lid-driven cavity, 128^3 hexahedra (2,097,152 cells),
Re = 1000, steady SIMPLE with CG+DILU for p and BiCGSTAB+DILU for U (itmax 100,
rtol 1e-3).  A step is one SIMPLE iteration (one launch of the persistent
device program) continuing from the previous step, the run starting from zero
fields as the case does.  K steps are timed in FP64 (`value`, the reference's
arithmetic) and then, from the same initial fields, in mixed precision (FP32
Krylov on FP64 assembly with FP64 residual refinement and dots); the line
carries both rates, their ratio and the relative L2 difference of every field
after the K steps.  The case's working set (about 2 GB) is far larger than the
126 MB L2, so steps run back to back without an L2 flush; the smaller 2D
workloads flush L2 (a 256 MiB write) between steps.  Each step is timed with
CUDA events on the library's stream; per-phase device time comes from the
library's phase timers (XCAL_FLAG_PHASE_TIMERS).

N > 1 runs N independent replicas (one per rank, weak scaling): a single case
does not shard, and there is no collective on the data path.

--impl reference times the CPU restatement of the reference (oracle/, one
thread, as the single-threaded reference) on the same mesh in the same cell
numbering, over the first outer iterations of the case (a bounded sample), and
prints the same metric.  That arm builds its mesh and numbering without the
product library.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "xcalibre_tw.jl_b200"))

METRIC = "SIMPLE cell-iters/s"
UNIT = "cell-iters/s"
RENUMBER = {"none": 0, "rcm": 1, "color": 2}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="xcal", choices=["xcal", "reference"])
    ap.add_argument("--config", default="cavity3d", choices=["bfs", "cavity", "cavity3d", "flatplate", "serve"])
    ap.add_argument("--serve-cases", type=int, default=512)
    ap.add_argument("--serve-rate", type=float, default=20.0, help="Poisson arrival rate, cases/s")
    ap.add_argument("--serve-nmax", type=int, default=400)
    ap.add_argument("--serve-maxit", type=int, default=3000, help="per-case SIMPLE iteration cap")
    ap.add_argument("--slots", type=int, default=512, help="serving: cases running at once")
    ap.add_argument("--tiles-per-cta", type=int, default=0, help="serving: CTA group sizing (0: library default)")
    ap.add_argument("--max-ctas", type=int, default=0, help="serving: largest CTA group (0: library default)")
    ap.add_argument("--serve-check", type=int, default=4, help="cases re-run alone for the parity check")
    ap.add_argument("--serve-seq", type=int, default=64,
                    help="cases of the stream, evenly spaced, also run one at a time on the whole-GPU path (0: skip)")
    ap.add_argument("--serve-seq-seconds", type=float, default=120.0,
                    help="time bound of the one-at-a-time sample")
    ap.add_argument("--precision-report", type=int, default=0, metavar="ITERS",
                    help="run ITERS SIMPLE iterations in FP64 and in mixed precision and report the "
                         "relative L2 difference of every field and both timings (one JSON line)")
    ap.add_argument("--renumber", default="color", choices=["color", "rcm", "none"])
    ap.add_argument("--size", type=int, default=None,
                    help="bfs: cells per step height (27); cavity: cells per side (40); cavity3d: cells per side (128)")
    ap.add_argument("--precision", default=None, choices=["both", "fp64", "mixed"],
                    help="both (cavity3d default): FP64 value and mixed beside it; fp64 (2D default); mixed")
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="CPU baseline sample budget (s)")
    ap.add_argument("--ref-seconds", type=float, default=60.0, help="--impl reference sample budget (s)")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-flush", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip xcal_autotune (the launch form of the library's heuristic is timed)")
    return ap.parse_args()


def build_case(name, size=None, mesh_builder=None):
    """(mesh, model, config, pref, description) of a named workload.  2D meshes
    are written as UNV by the seeded generator and read by mesh_builder (the
    library's builder by default)."""
    from xcal import cases, meshgen
    if name == "bfs":
        size = size or 27
        mesh = mesh_builder(cases._unv("bfs", meshgen.bfs_unv, cells_per_h=size)) if mesh_builder else None
        mesh, model, config, pref = cases.bfs(size, iterations=2000, mesh=mesh)
        desc = f"laminar backward-facing step h=10mm, {size} cells/h, graded 1.05, jittered 10%, Re=50"
    elif name == "cavity":
        size = size or 40
        mesh = mesh_builder(cases._unv("cavity", meshgen.cavity_unv, n=size, L=0.1)) if mesh_builder else None
        mesh, model, config, pref = cases.cavity2d(size, iterations=1000, mesh=mesh)
        desc = f"2D lid-driven cavity {size}x{size}, Re=100"
    elif name == "flatplate":
        nx, ny = (size or 600), (size or 600) * 5 // 12
        mesh = mesh_builder(cases._unv("flatplate", meshgen.flatplate_unv, nx=nx, ny=ny)) if mesh_builder else None
        mesh, model, config, pref = cases.flatplate(nx, ny, iterations=3000, mesh=mesh)
        desc = f"k-omega flat plate 1 m x 0.2 m, {nx}x{ny} graded quads, U=10 m/s, nu=1.5e-5"
    else:
        size = size or 128
        mesh, model, config, pref = cases.cavity3d(size, iterations=500)
        desc = f"3D lid-driven cavity {size}^3 hexahedra, Re=1000, 500-iteration case"
    return mesh, model, config, pref, desc


# ------------------------------------------------------------ byte model
def byte_model(mesh, kry, ns, sk=8):
    """Algorithmic HBM bytes of one SIMPLE iteration per phase class
    (xcal._abi.PHASES) given its Krylov counts (kry: U iterations per
    component, p iterations at index 3); sk is the value size of the Krylov
    iterations (8 FP64, 4 mixed).  Each phase class counts the minimum traffic
    of its operations: every array it must read or write once.  Per-operation
    figures (s value size, k right-hand sides):
      SpMV (CSR)              nnz*(s+4) + (N+1)*4 + 2*k*N*s
      DILU apply (2 sweeps)   2*Fi*(s+4) + 2*N*s + 4*k*N*s
      DILU update             Fi*(2s+4) + 2*N*s
      vector phase            (vectors read + written) * k * N * s
      assembly (k RHS)        Fi*(8+6s) + N*(5s + 3s*(k-1)) + Fb*(4+4s)
      face phase              face arrays * F * s + gathered cell arrays * N * s
    """
    s = 8
    N, F, Fb = mesh.ncells, mesh.nfaces, mesh.nbfaces
    Fi = F - Fb
    nnz = N + 2 * Fi

    def spmv(k, v):
        return nnz * (v + 4) + (N + 1) * 4 + 2 * k * N * v

    def spmv_mat(v):
        return nnz * (v + 4) + (N + 1) * 4

    def dilu(k, v):
        return 2 * Fi * (v + 4) + 2 * N * v + 4 * k * N * v

    def dilu_upd(v):
        return Fi * (2 * v + 4) + 2 * N * v

    itU = int(max(kry[:ns]))
    itP = int(kry[3])
    mixed_copy = nnz * sk if sk != 8 else 0
    B = {}
    B["setup"] = 0
    B["momentum_assembly"] = (Fi * (8 + 6 * s) + N * (5 * s + 3 * s * (ns - 1)) + Fb * (4 + 4 * s) + spmv(ns, s)
                              + mixed_copy + 3 * ns * N * sk)
    B["pressure_assembly"] = (F * s * ns + N * 2 * s + Fi * (8 + 4 * s) + N * 3 * s + spmv(1, s) + mixed_copy
                              + 3 * N * sk)
    B["precon_setup"] = dilu_upd(sk) + dilu(ns, sk) + 2 * ns * N * sk + dilu_upd(sk) + dilu(1, sk) + 2 * N * sk
    # BiCGSTAB: phases A (p recomputed from r, p, v; q, p, M^-1 level 0 out) and D
    # (s from r, v; x += alpha p; q, s, t out); CG: phase A (p from z, p; p, q out)
    B["krylov_spmv"] = (itU * (2 * spmv_mat(sk) + 14 * ns * N * sk) + itP * (spmv_mat(sk) + 4 * N * sk))
    # BiCGSTAB: two M^-1 applications with their dots; CG: x/r update + M^-1 + <r,z>
    B["krylov_precon"] = itU * (2 * dilu(ns, sk) + 4 * ns * N * sk) + itP * (dilu(1, sk) + 9 * N * sk)
    B["krylov_vector"] = itU * 7 * ns * N * sk
    B["residual"] = spmv(ns, s) + 5 * ns * N * s + spmv(1, s) + N * s
    B["face"] = ((F * s * (1 + ns) + F * 16 + (1 + ns) * N * s)      # rDf, Uf(H)
                 + (F * s + F * 16 + N * s)                         # pf
                 + (F * s * (1 + ns) + F * 16 + ns * N * s + F * s))  # Uf(U), flux!
    B["gradient"] = Fi * (4 + 1) * 2 + F * s * (2 + ns) + N * s + ns * N * s + 3 * ns * N * s
    B["update"] = ns * N * (sk + 2 * s) + N * (sk + 2 * s)
    B["turbulence"] = 0
    return B


# ------------------------------------------------------------------ clocks
class ClockSampler:
    def __init__(self, gpu_index):
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"xcal_clocks_{os.getpid()}.csv")
        self.gpu = gpu_index

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.strip()]
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        mx = float(rows[0][2])
        reasons = set()
        for r in rows:
            names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(rows)}


def load_peaks():
    try:
        m = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic(workload_key):
    try:
        t = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        return t.get(workload_key)
    except Exception:
        return None




# ------------------------------------------------------------- CPU oracle
def oracle_case(a, renumber):
    """The workload for the CPU restatement, built without the product library:
    2D meshes through the oracle's own UNV builder, the cell numbering of the
    device path through the oracle's permutation (oracle.renumbered)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    mesh, model, config, pref, desc = build_case(a.config, a.size, mesh_builder=lambda p: O.build_unv(p).to_mesh2())
    dev_mesh, perm = O.renumbered(mesh, renumber)
    return mesh, model, config, pref, desc, dev_mesh, perm


def cpu_oracle_rate(model, config, pref, dev_mesh, perm, seconds, per_iter_hint=None):
    """Single-threaded CPU restatement of the reference on the same mesh in the
    device's cell numbering: SIMPLE iterations from the start of the case,
    as many as fit the budget (at least 1), loop time only (set-up excluded)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import xcal as X
    from xcal import cases
    om = O.from_mesh2(dev_mesh)
    case, keep = X.make_case(model, config, pref)
    U, p = cases.fields(model)
    Ud = np.zeros_like(U)
    pd = np.zeros_like(p)
    Ud[:, perm] = U
    pd[perm] = p
    extra = {}
    if X.isturbulent(model):
        t = model.turbulence
        for name, f in (("k", t.k.values), ("omega", t.omega.values), ("nut", t.nut.values)):
            v = np.zeros_like(p)
            v[perm] = f
            extra[name] = v
    if per_iter_hint is None:
        out = O.run(om, case, 1, Ud, pd, ref_cell=int(perm[0]), **extra)
        per = out["loop_seconds"]
        if per >= 0.5 * seconds:
            return dev_mesh.ncells * out["done"] / per, out["done"], per
    else:
        per = per_iter_hint
    its = max(1, min(3000, int(seconds / max(per, 1e-6))))
    out = O.run(om, case, its, Ud, pd, ref_cell=int(perm[0]), **extra)
    dt = out["loop_seconds"]
    return dev_mesh.ncells * out["done"] / dt, out["done"], dt


def cpu_model():
    try:
        for l in open("/proc/cpuinfo"):
            if l.startswith("model name"):
                return l.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"



# ----------------------------------------------------------------- serving
def run_alone(c, precision, maxit, tol=1e-6):
    """One case through the plain path: its own context, whole-GPU launch
    (grid barrier over every resident CTA), stop at `tol` or `maxit`, stop at
    a non-finite Krylov norm; timed from context creation to the fields read
    back (the calls a caller makes per case).  Returns (iterations, status,
    seconds, U, p)."""
    import xcal as X
    from xcal import _abi, cases
    lib = _abi.load()
    t0 = time.perf_counter()
    case, keep = X.make_case(c["model"], c["config"], c["pref"], precision)
    s = X.Solver(c["mesh"], renumber=_abi.RENUMBER_COLOR, flags=_abi.FLAG_ABORT_ON_NAN)
    s.setup(case)
    s.set_tolerance(tol)
    U0, p0 = cases.fields(c["model"])
    for f, v in ((_abi.FIELD_UX, U0[0]), (_abi.FIELD_UY, U0[1]), (_abi.FIELD_UZ, U0[2]), (_abi.FIELD_P, p0)):
        s.set_field(f, v)
    R = np.ones((4, maxit))
    done = np.zeros(1, dtype=np.int32)
    st = lib.xcal_simple_run(s.ctx, maxit, _abi.dptr(R[0]), _abi.dptr(R[1]), _abi.dptr(R[2]),
                             _abi.dptr(R[3]), None, _abi.i32ptr(done))
    if st not in (0, -5):   # XCAL_ERR_NAN: diverged and stopped, as in the serving loop
        _abi.check(st, s.ctx, "xcal_simple_run")
    U = np.stack([s.get_field(f) for f in (_abi.FIELD_UX, _abi.FIELD_UY, _abi.FIELD_UZ)])
    p = s.get_field(_abi.FIELD_P)
    s.close()
    return int(done[0]), st, time.perf_counter() - t0, U, p


def serve_one_at_a_time(a, stream):
    """The same stream one case at a time on the plain FP64 path: every
    (len/serve_seq)-th case (evenly spaced), the same tolerance, cap and stop
    on a non-finite norm as the serving loop.  One untimed case first loads
    the program."""
    from xcal import _abi
    run_alone(stream[0], _abi.PREC_FP64, 5)
    t_all, cells_its, count, conv = 0.0, 0.0, 0, 0
    stride = max(1, len(stream) // a.serve_seq)
    for k in range(0, stride * min(a.serve_seq, len(stream)), stride):
        if t_all > a.serve_seq_seconds:
            break
        its, st, dt, U, p = run_alone(stream[k], _abi.PREC_FP64, a.serve_maxit)
        t_all += dt
        cells_its += stream[k]["mesh"].ncells * its
        count += 1
        conv += int(st == 0 and its < a.serve_maxit)
    return {"cases": count, "every": stride, "cases_per_s": count / t_all, "converged_cases_per_s": conv / t_all,
            "cell_iters_per_s": cells_its / t_all, "seconds": t_all,
            "launch": "plain path, FP64, whole-GPU grid launch, one case at a time"}


def serve_main(a):
    """Serving stream: Poisson arrivals of independent cavity/BFS cases, each
    run to residuals <= 1e-6 in mixed precision by the library's serving loop
    (xcal_serve_*: one persistent launch, a CTA group per case, admission by
    device footprint); cases/s and time-to-converged percentiles, the same
    stream one case at a time on the plain FP64 path, and a parity sample of
    cases re-run alone (mixed: bitwise; FP64: relative L2)."""
    import xcal as X
    from xcal import _abi, cases
    if int(os.environ.get("RANK", "0")) != 0:
        return
    stream = cases.serving_stream(a.serve_cases, rate=a.serve_rate, nmax=a.serve_nmax)
    srv = X.Server(slots=a.slots, max_iterations=a.serve_maxit, tolerance=1e-6, precision=_abi.PREC_MIXED,
                   tiles_per_cta=a.tiles_per_cta, max_ctas=a.max_ctas)
    pending, results = {}, {}
    t0 = time.perf_counter()
    t_last = t0

    def drain(wait_ms):
        nonlocal t_last
        for k in list(pending):
            r = srv.poll(pending[k], wait_ms=wait_ms)
            if r is not None:
                results[k] = r
                del pending[k]
                t_last = time.perf_counter()
                wait_ms = 0
    with ClockSampler(0) as clk:
        for k, c in enumerate(stream):
            while time.perf_counter() - t0 < c["t"]:
                drain(0)
                time.sleep(0.0005)
            pending[k] = srv.submit(c["model"], c["config"], c["pref"])
        while pending:
            drain(20)
    st = srv.stats()
    srv.close()
    wall = t_last - t0
    ks = sorted(results)
    ok = {k: results[k]["status"] == 0 for k in ks}
    conv = {k: ok[k] and results[k]["converged"] == 1 for k in ks}
    diverged = {k: results[k]["status"] == -5 for k in ks}
    lat = np.array([results[k]["total_ms"] for k in ks if conv[k]] or [np.nan])
    # parity sample: the smallest and the largest converged case of each kind
    pick = []
    for kind in ("cavity", "bfs"):
        cand = sorted([k for k in ks if conv[k] and stream[k]["kind"] == kind], key=lambda k: stream[k]["mesh"].ncells)
        pick += cand[:1] + cand[-1:] if cand else []
    check = []
    for k in pick[: a.serve_check]:
        c, r = stream[k], results[k]
        row = {"case": f"{c['kind']} N={c['N']} cells={c['mesh'].ncells} Re={c['Re']:.0f}",
               "iterations_served": r["iterations"]}
        its, stt, dt, U, p = run_alone(c, _abi.PREC_MIXED, a.serve_maxit)
        row["alone_mixed"] = {"iterations": its, "bitwise_equal": bool(its == r["iterations"] and
                                                                      np.array_equal(U, r["U"]) and
                                                                      np.array_equal(p, r["p"]))}
        its, stt, dt, U, p = run_alone(c, _abi.PREC_FP64, a.serve_maxit)
        d = float(max(np.linalg.norm(U[i] - r["U"][i]) / max(np.linalg.norm(U[i]), 1e-300) for i in range(2)))
        row["alone_fp64"] = {"iterations": its, "U_rel_l2": d}
        check.append(row)
    seq = serve_one_at_a_time(a, stream) if a.serve_seq > 0 else None
    value = len(results) / wall
    nconv = int(sum(conv.values()))
    cit = st["cell_iterations"] / wall
    line = {
        "metric": "serving cases/s", "value": value, "unit": "cases/s", "n_gpus": 1,
        "steps": len(stream), "warmup": 0, "ms_per_step": 1000.0 * wall / max(len(results), 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
        "data": "synthetic cases from the seeded serving generator (numpy default_rng(12345))",
        "config": {"workload": f"{len(stream)} cavity/BFS cases, Poisson {a.serve_rate}/s, N in [40,{a.serve_nmax}], "
                               f"Re U(50,1000), stop at residuals <= 1e-6 (cap {a.serve_maxit})",
                   "slots": a.slots, "precision": "mixed",
                   "launch": f"one persistent launch of {st['grid_ctas']} CTAs, a CTA group per case",
                   "device_arena_bytes": st["device_bytes"], "device_arena_peak_bytes": st["device_bytes_peak"]},
        "time_to_converged_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                                 "max": float(np.max(lat)), "over": "converged cases, submit to result"},
        "finished": len(results), "converged": nconv, "capped": int(sum(ok.values()) - nconv),
        "diverged": int(sum(diverged.values())), "failed_other": int(st["failed"] - sum(diverged.values())),
        "converged_cases_per_s": nconv / wall,
        "note": "value = finished cases (converged, capped or diverged) / wall time; diverged = non-finite "
                "Krylov norms, stopped early (the reference SIMPLE diverges on BFS above Re ~100-150)",
        "cell_iters_per_s": cit, "wall_s": wall,
        "one_at_a_time": seq,
        "vs_one_at_a_time": None if not seq else {
            "cases_per_s": value / seq["cases_per_s"],
            "converged_cases_per_s": (nconv / wall) / max(seq["converged_cases_per_s"], 1e-300),
            "cell_iters_per_s": cit / seq["cell_iters_per_s"],
            "note": "the whole stream served (mixed) against an evenly spaced sample of it run one at a time "
                    "on the plain FP64 path"},
        "mean_ms": {k: float(np.mean([results[j][k] for j in results])) for k in ("queue_ms", "setup_ms", "run_ms")},
        "parity_sample": check, "clocks": clk.summary(), "impl": "xcal",
    }
    print(json.dumps(line))


# -------------------------------------------------------- precision report
def precision_report(a):
    """FP64 and mixed precision from the same initial fields, ITERS iterations
    each; relative L2 of the mixed fields against the FP64 ones."""
    import xcal as X
    from xcal import _abi, cases
    mesh, model, config, pref, desc = build_case(a.config, a.size)
    its = a.precision_report
    out = {}
    for name, prec in (("fp64", _abi.PREC_FP64), ("mixed", _abi.PREC_MIXED)):
        case, keep = X.make_case(model, config, pref, prec)
        s = X.Solver(mesh, renumber=_abi.RENUMBER_COLOR)
        s.setup(case)
        U0, p0 = cases.fields(model)
        for f, v in ((_abi.FIELD_UX, U0[0]), (_abi.FIELD_UY, U0[1]), (_abi.FIELD_UZ, U0[2]), (_abi.FIELD_P, p0)):
            s.set_field(f, v)
        r = s.run(its, want_krylov=True)
        fields = {k: s.get_field(f) for k, f in (("Ux", _abi.FIELD_UX), ("Uy", _abi.FIELD_UY), ("Uz", _abi.FIELD_UZ),
                                                  ("p", _abi.FIELD_P))}
        out[name] = dict(ms=s.last_ms(), done=r["done"], fields=fields,
                         R_last=[float(r[k][r["done"] - 1]) for k in ("R_ux", "R_uy", "R_uz", "R_p")],
                         kry=r["krylov"][: r["done"]].mean(axis=0).tolist())
        s.close()
    rel = {k: float(np.linalg.norm(out["mixed"]["fields"][k] - out["fp64"]["fields"][k]) /
                    max(np.linalg.norm(out["fp64"]["fields"][k]), 1e-300)) for k in ("Ux", "Uy", "Uz", "p")}
    print(json.dumps({"metric": "mixed vs fp64 relative L2", "config": {"workload": desc, "cells": mesh.ncells,
                      "iterations": its}, "rel_l2": rel,
                      "fp64": {k: v for k, v in out["fp64"].items() if k != "fields"},
                      "mixed": {k: v for k, v in out["mixed"].items() if k != "fields"},
                      "speedup": out["fp64"]["ms"] / out["mixed"]["ms"]}))


# ------------------------------------------------------------------- ranks
def init_ranks(world, local, backend="nccl", timeout_s=120):
    """One process per GPU: set the device and join the process group (None
    for a single rank).  The group carries only the timing barrier and the
    max-over-ranks reduction, never case data."""
    if world <= 1:
        return None
    import datetime
    import torch
    import torch.distributed as dist
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, init_method="env://", timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(x, dist, device):
    """The largest per-rank value (the slowest replica sets the job's time)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, units_per_rank, seconds):
    """Whole-job rate: every rank processed units_per_rank in at most `seconds`."""
    return world * units_per_rank / seconds


# -------------------------------------------------------------------- main
def reference_main(a, rank):
    """--impl reference: the CPU restatement (one thread) on the workload's mesh
    in the device's numbering, a bounded sample of the case's first outer
    iterations.  Rank 0 alone runs under torchrun."""
    if rank != 0:
        return
    mode = RENUMBER[a.renumber]
    mesh, model, config, pref, desc, dev_mesh, perm = oracle_case(a, mode)
    rate, its, dt = cpu_oracle_rate(model, config, pref, dev_mesh, perm, a.ref_seconds)
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": a.gpus,
            "steps": its, "warmup": 0, "ms_per_step": 1000 * dt / its, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic mesh from the seeded generator (reference construction rules)",
            "config": {"workload": desc, "cells": mesh.ncells, "renumber": a.renumber,
                       "same_config": True, "sample": f"first {its} SIMPLE iterations"},
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": f"first {its} SIMPLE iterations of the case ({dt:.1f} s loop time, "
                                       f"set-up excluded), 1 thread (the reference is single-threaded), "
                                       f"CPU: {cpu_model()}"},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_timed(s, steps, dist, dev, flush, clk=None):
    """K SIMPLE iterations, one launch each, event-timed on the library's
    stream; returns per-step ms, Krylov counts and the phase timers' sums."""
    import torch
    from xcal import _abi
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ms, kry = [], []
    ph = {k: [0.0, 0] for k in _abi.PHASES}
    for _ in range(steps):
        if flush is not None:
            flush.fill_(1.0)
            torch.cuda.synchronize(dev)
        out = s.run(1)
        ms.append(s.last_ms())
        kry.append(out["krylov"][0])
        for k, (cyc, cnt) in s.last_phases().items():
            ph[k][0] += cyc
            ph[k][1] += cnt
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    return np.array(ms), np.array(kry), ph


def phase_table(mesh, ns, sk, ms, kry, ph, peak):
    """Per phase class: device time (the timers' cycle shares of the event-timed
    total), algorithmic bytes (byte_model with the measured Krylov counts) and
    the achieved fraction of the HBM peak."""
    from xcal import _abi
    bytes_ = {k: 0.0 for k in _abi.PHASES}
    for kr in kry:
        for k, v in byte_model(mesh, kr, ns, sk).items():
            bytes_[k] += v
    total_cyc = sum(v[0] for v in ph.values())
    total_ms = float(ms.sum())
    out = {}
    for k in _abi.PHASES:
        cyc, cnt = ph[k]
        if cnt == 0:
            continue
        t = total_ms * cyc / total_cyc if total_cyc > 0 else 0.0
        gbs = bytes_[k] / (t / 1000.0) / 1e9 if t > 0 else None
        out[k] = {"ms_per_step": t / len(ms), "phases_per_step": cnt / len(ms),
                  "us_per_phase": 1000.0 * t / cnt, "share": t / total_ms,
                  "algorithmic_bytes_per_step": bytes_[k] / len(ms),
                  "achieved_gbs": gbs, "frac_of_peak": (gbs / peak) if gbs else None}
    return out, float(sum(bytes_.values()))


def main():
    a = parse()
    if a.precision_report:
        return precision_report(a)
    if a.config == "serve":
        if a.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving loop "
                                                                   "(one case per Julia process)"}))
            return
        return serve_main(a)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        return reference_main(a, rank)
    precision = a.precision or ("both" if a.config == "cavity3d" else "fp64")

    import torch
    dist = init_ranks(world, local)
    import xcal as X
    from xcal import _abi, cases

    mesh, model, config, pref, desc = build_case(a.config, a.size)
    N = mesh.ncells
    ns = 3 if mesh.dim == 3 else 2
    renum = RENUMBER[a.renumber]
    dev = torch.device("cuda", local if world > 1 else 0)
    U0, p0 = cases.fields(model)
    turb = [(_abi.FIELD_K, model.turbulence.k.values.copy()), (_abi.FIELD_OMEGA, model.turbulence.omega.values.copy()),
            (_abi.FIELD_NUT, model.turbulence.nut.values.copy())] if X.isturbulent(model) else []
    # inputs larger than L2 need no flush between steps; smaller workloads flush
    big = N * 8 * 20 > 4 * 126 * 2 ** 20
    flush = None if (a.no_flush or big) else torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def reset(s):
        for f, v in ((_abi.FIELD_UX, U0[0]), (_abi.FIELD_UY, U0[1]), (_abi.FIELD_UZ, U0[2]), (_abi.FIELD_P, p0)):
            s.set_field(f, v)
        for f, v in turb:
            s.set_field(f, v)

    peak, peak_kind = load_peaks()
    gpu_index = local if world > 1 else int(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0] or 0)
    runs = {}
    precs = [("fp64", _abi.PREC_FP64), ("mixed", _abi.PREC_MIXED)]
    if precision != "both":
        precs = [p for p in precs if p[0] == precision]
    clocks = None
    solver_keep = None
    for name, prec in precs:
        case, keep = X.make_case(model, config, pref, prec)
        s = X.Solver(mesh, device=local if world > 1 else 0, renumber=renum, flags=_abi.FLAG_PHASE_TIMERS)
        s.setup(case)
        reset(s)
        # the library's autotuner picks the launch form (untimed set-up; every
        # form computes the same values)
        tune = None if a.no_tune else s.autotune(3)
        for _ in range(max(a.warmup, 0)):
            s.run(1, want_krylov=False)
        reset(s)
        with ClockSampler(gpu_index) as clk:
            ms, kry, ph = run_timed(s, a.steps, dist, dev, flush)
        if clocks is None:
            clocks = clk.summary()
        fields = {k: s.get_field(f) for k, f in (("Ux", _abi.FIELD_UX), ("Uy", _abi.FIELD_UY),
                                                  ("Uz", _abi.FIELD_UZ), ("p", _abi.FIELD_P))}
        total_ms = max_over_ranks(float(ms.sum()), dist, dev)
        sk = 4 if prec == _abi.PREC_MIXED else 8
        table, total_bytes = phase_table(mesh, ns, sk, ms, kry, ph, peak)
        runs[name] = dict(ms=ms, kry=kry, total_ms=total_ms, fields=fields, phases=table, tune=tune,
                          bytes_per_step=total_bytes / a.steps,
                          value=job_throughput(world, N * a.steps, total_ms / 1000.0))
        if solver_keep is None:
            solver_keep = (s, keep)
        else:
            s.close()
    main_name = precs[0][0]
    R = runs[main_name]
    s, _keep = solver_keep

    # end to end through the public API with host buffers (the first precision)
    e2e_steps = a.e2e_steps or min(a.steps, 30)
    reset(s)
    Uh = [U0[0].copy(), U0[1].copy(), U0[2].copy()]
    ph_ = p0.copy()
    fset = [(_abi.FIELD_UX, 0), (_abi.FIELD_UY, 1)] + ([(_abi.FIELD_UZ, 2)] if ns == 3 else [])
    if dist:
        dist.barrier()
    e2e_t = 0.0
    for _ in range(e2e_steps):
        if flush is not None:
            flush.fill_(1.0)
            torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for f, d in fset:
            s.set_field(f, Uh[d])
        s.set_field(_abi.FIELD_P, ph_)
        s.run(1, want_krylov=False)
        for f, d in fset:
            Uh[d] = s.get_field(f)
        ph_ = s.get_field(_abi.FIELD_P)
        e2e_t += time.perf_counter() - t0
    e2e_value = job_throughput(world, N * e2e_steps, max_over_ranks(e2e_t, dist, dev))
    h2d = (len(fset) + 1) * N * 8
    d2h = (len(fset) + 1) * N * 8 + 4 * 8 + 5 * 4
    s.close()

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        mesh_o, model_o, config_o, pref_o, desc_o, dev_mesh, perm = oracle_case(a, renum)
        rate, its, dt = cpu_oracle_rate(model_o, config_o, pref_o, dev_mesh, perm, a.cpu_seconds)
        cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"CPU oracle on the same mesh and numbering, first {its} SIMPLE iterations "
                         f"({dt:.1f} s loop time), 1 thread, {cpu_model()}"}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    frac = R["bytes_per_step"] * a.steps / (R["total_ms"] / 1000.0) / 1e9
    line = {
        "metric": METRIC, "value": R["value"], "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": R["total_ms"] / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if main_name == "fp64" else "f64+f32",
        "data": "synthetic mesh from the seeded generator (reference construction rules)",
        "config": {"workload": desc, "cells": N, "renumber": a.renumber, "precision": main_name,
                   "step": "one SIMPLE iteration, continuing from the previous step (run from zero fields)",
                   "l2": ("not flushed: working set larger than L2" if flush is None and big else
                          "flushed between steps (256 MiB write)" if flush is not None else "not flushed"),
                   "krylov_mean": {"U": float(R["kry"][:, 0].mean()), "p": float(R["kry"][:, 3].mean())},
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": frac, "peak": peak, "unit": "GB/s", "frac": frac / peak,
                     "peak_kind": peak_kind, "traffic": load_traffic(f"{a.config}_{N}_{main_name}_simple"),
                     "kernel": "xcal_program_kernel (persistent SIMPLE iteration)"},
        "phases": {k: v["phases"] for k, v in runs.items()},
        "autotune": {k: v["tune"] for k, v in runs.items()},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps, "precision": main_name},
        "gpu_launches": a.steps,
        "clocks": clocks,
        "impl": "xcal",
    }
    if "mixed" in runs and "fp64" in runs:
        m, f = runs["mixed"], runs["fp64"]
        keys = ("Ux", "Uy", "Uz", "p") if ns == 3 else ("Ux", "Uy", "p")
        rel = {k: float(np.linalg.norm(m["fields"][k] - f["fields"][k]) / max(np.linalg.norm(f["fields"][k]), 1e-300))
               for k in keys}
        mfrac = m["bytes_per_step"] * a.steps / (m["total_ms"] / 1000.0) / 1e9
        line["mixed"] = {"value": m["value"], "unit": UNIT, "ms_per_step": m["total_ms"] / a.steps,
                         "speedup_vs_fp64": m["value"] / f["value"],
                         "rel_l2_vs_fp64_after_steps": rel,
                         "krylov_mean": {"U": float(m["kry"][:, 0].mean()), "p": float(m["kry"][:, 3].mean())},
                         "roofline_frac": mfrac / peak,
                         "dtype": "f32 Krylov vectors/matrix/DILU; f64 assembly, residual b-Ax, dots"}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
