"""Benchmark: SIMPLE cell-iterations/s of the laminar backward-facing step
(47,385 cells, FP64, CG+DILU for p, BiCGSTAB+DILU for U) on the device path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl xcal|reference]
                    [--config bfs|cavity|cavity3d] [--renumber color|rcm|none]

A step is one SIMPLE iteration of the case (one launch of the persistent device
program).  Steps run from zero initial fields, as the case does; L2 is flushed
between steps (a 256 MiB write), and each step is timed with CUDA events on the
library's stream.  N > 1 runs N independent replicas (one per rank, weak
scaling): a single case does not shard, there is no collective on the data path.

--impl reference times the CPU restatement of the reference (single thread, as
the reference) on the same case and prints the same metric.
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="xcal", choices=["xcal", "reference"])
    ap.add_argument("--config", default="bfs", choices=["bfs", "cavity", "cavity3d", "flatplate", "serve"])
    ap.add_argument("--serve-cases", type=int, default=512)
    ap.add_argument("--serve-rate", type=float, default=20.0, help="Poisson arrival rate, cases/s")
    ap.add_argument("--serve-nmax", type=int, default=400)
    ap.add_argument("--serve-maxit", type=int, default=3000, help="per-case SIMPLE iteration cap")
    ap.add_argument("--slots", type=int, default=30,
                    help="concurrent serving cases (<= 30: one hardware work queue per worker)")
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
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="mixed: FP32 Krylov on FP64 assembly with FP64 residual refinement")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-flush", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


def build_case(name, size=None):
    from xcal import cases
    if name == "bfs":
        size = size or 27
        mesh, model, config, pref = cases.bfs(size, iterations=2000)
        desc = f"laminar backward-facing step h=10mm, {size} cells/h, graded 1.05, jittered 10%, Re=50"
    elif name == "cavity":
        size = size or 40
        mesh, model, config, pref = cases.cavity2d(size, iterations=1000)
        desc = f"2D lid-driven cavity {size}x{size}, Re=100"
    elif name == "flatplate":
        nx, ny = (size or 600), (size or 600) * 5 // 12
        mesh, model, config, pref = cases.flatplate(nx, ny, iterations=3000)
        desc = f"k-omega flat plate 1 m x 0.2 m, {nx}x{ny} graded quads, U=10 m/s, nu=1.5e-5"
    else:
        size = size or 128
        mesh, model, config, pref = cases.cavity3d(size, iterations=500)
        desc = f"3D lid-driven cavity {size}^3 hexahedra, Re=1000"
    return mesh, model, config, pref, desc


# ------------------------------------------------------------ byte model
def algorithmic_bytes(mesh, kry, ns, sk=8):
    """Algorithmic HBM bytes of one SIMPLE iteration given its Krylov counts
    (U iterations per component, p iterations); sk is the size of the Krylov
    iterations' matrix and vector values (8, or 4 in mixed precision).
    Per-operation figures (s the value size):
      SpMV (CSR, k vectors)   nnz*(s+4) + (N+1)*4 + 2*k*N*s
      DILU apply (k vectors)  2*Fi*(s+4) + 2*N*s + 4*k*N*s
      DILU update             Fi*(2s+4) + 2*N*s
      vector kernels          (vectors read + written) * N * s
      assembly (k RHS)        Fi*(8+6s) + N*(5s + 3s*(k-1)) + Fb*(4+4s)
      face fields             face arrays * F * s + gathered cell arrays * N * s
    """
    s = 8
    N = mesh.ncells
    F = mesh.nfaces
    Fb = mesh.nbfaces
    Fi = F - Fb
    nnz = N + 2 * Fi

    def spmv(k, s=s):
        return nnz * (s + 4) + (N + 1) * 4 + 2 * k * N * s

    def dilu(k, s=s):
        return 2 * Fi * (s + 4) + 2 * N * s + 4 * k * N * s
    dilu_upd = Fi * (2 * s + 4) + 2 * N * s
    vec = N * s
    veck = N * sk
    itU = int(max(kry[:ns]))
    itP = int(kry[3])
    b = 0
    # momentum: assembly, r0 = b - A x0, DILU update + first apply, BiCGSTAB init
    b += Fi * (8 + 6 * s) + N * (5 * s + 3 * s * (ns - 1)) + Fb * (4 + 4 * s)
    b += spmv(ns) + dilu_upd + dilu(ns) + 3 * ns * vec
    b += itU * (2 * spmv(ns, sk) + 2 * dilu(ns, sk) + 20 * ns * veck)
    b += 3 * ns * vec                                    # x + x0
    b += spmv(ns) + (2 + 2) * ns * vec + N * (s + 4)     # residual!, remove_pressure_source!, H!
    b += F * s * (1 + ns) + (1 + ns) * N * s + F * 8     # rDf, Uf(H) face interpolation
    # pressure: div!, assembly, CG
    b += F * s * ns + N * 2 * s + Fi * (8 + 4 * s) + N * 3 * s
    b += spmv(1) + dilu_upd + dilu(1) + 3 * vec
    b += itP * (spmv(1, sk) + dilu(1, sk) + 13 * veck)
    b += 3 * vec + spmv(1) + 2 * vec                     # relax, residual!
    b += F * s + 2 * N * s                               # pf interpolation
    b += Fi * (8 + 2 * s) + N * s * (1 + ns * 3)         # Green-Gauss + correct_velocity!
    b += F * s * (1 + 3) + ns * N * s                    # Uf(U), flux!
    return b


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
def cpu_oracle_rate(mesh, model, config, pref, seconds):
    """Single-threaded CPU restatement of the reference on the same case: time
    SIMPLE iterations from the start of the run until the budget is used."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import xcal as X
    from xcal import cases
    om = O.from_mesh2(mesh)
    case, keep = X.make_case(model, config, pref)
    U, p = cases.fields(model)
    t0 = time.perf_counter()
    O.run(om, case, 2, U, p)                 # estimate
    per = (time.perf_counter() - t0) / 2
    its = max(2, min(2000, int(seconds / max(per, 1e-6))))
    t0 = time.perf_counter()
    out = O.run(om, case, its, U, p)
    dt = time.perf_counter() - t0
    its_done = out["done"]
    return mesh.ncells * its_done / dt, its_done, dt


def cpu_model():
    try:
        for l in open("/proc/cpuinfo"):
            if l.startswith("model name"):
                return l.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


# ----------------------------------------------------------------- serving
def serve_one_at_a_time(a, stream, served):
    """Every (len/serve_seq)-th case of the same stream run one at a time on the plain path: one
    context per case with the whole-GPU launch (grid barrier over all SMs),
    mixed precision, the same tolerance, cap and stop on a non-finite Krylov
    norm as the serving loop.  Each case is timed from context creation to
    its fields read back, the calls a caller makes per case.  One untimed
    case first loads the program."""
    import xcal as X
    from xcal import _abi, cases
    lib = _abi.load()
    maxit = a.serve_maxit

    def one(c):
        case, keep = X.make_case(c["model"], c["config"], c["pref"], _abi.PREC_MIXED)
        s = X.Solver(c["mesh"], renumber=_abi.RENUMBER_COLOR, flags=_abi.FLAG_ABORT_ON_NAN)
        s.setup(case)
        s.set_tolerance(1e-6)
        U0, p0 = cases.fields(c["model"])
        for f, v in ((_abi.FIELD_UX, U0[0]), (_abi.FIELD_UY, U0[1]), (_abi.FIELD_UZ, U0[2]), (_abi.FIELD_P, p0)):
            s.set_field(f, v)
        R = np.ones((4, maxit))
        done = np.zeros(1, dtype=np.int32)
        st = lib.xcal_simple_run(s.ctx, maxit, _abi.dptr(R[0]), _abi.dptr(R[1]), _abi.dptr(R[2]),
                                 _abi.dptr(R[3]), None, _abi.i32ptr(done))
        if st not in (0, -5):   # XCAL_ERR_NAN: diverged and stopped, as in the serving loop
            _abi.check(st, s.ctx, "xcal_simple_run")
        if st == 0:
            for f in (_abi.FIELD_UX, _abi.FIELD_UY, _abi.FIELD_UZ, _abi.FIELD_P):
                s.get_field(f)
        s.close()
        return int(done[0])

    one(stream[0])
    t_all, cells_its, same, count = 0.0, 0.0, 0, 0
    stride = max(1, len(stream) // a.serve_seq)
    for k in range(0, stride * min(a.serve_seq, len(stream)), stride):
        if t_all > a.serve_seq_seconds:
            break
        t0 = time.perf_counter()
        its = one(stream[k])
        t_all += time.perf_counter() - t0
        cells_its += stream[k]["mesh"].ncells * its
        same += int(k in served and served[k]["iterations"] == its)
        count += 1
    return {"cases": count, "every": stride, "cases_per_s": count / t_all, "cell_iters_per_s": cells_its / t_all,
            "seconds": t_all, "iterations_equal_to_served": same,
            "launch": "whole-GPU grid launch, one case at a time, mixed precision"}


def serve_main(a):
    """Serving stream: Poisson arrivals of independent cavity/BFS cases, each
    run to residuals <= 1e-6 in mixed precision by the library's serving loop
    (xcal_serve_*); cases/s and time-to-converged percentiles, plus a parity
    sample of cases re-run alone (same precision: bitwise; FP64: rel. L2)."""
    import xcal as X
    from xcal import _abi, cases
    if int(os.environ.get("RANK", "0")) != 0:
        return
    stream = cases.serving_stream(a.serve_cases, rate=a.serve_rate, nmax=a.serve_nmax)
    srv = X.Server(slots=a.slots, max_iterations=a.serve_maxit, tolerance=1e-6)
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
                time.sleep(0.001)
            pending[k] = srv.submit(c["model"], c["config"], c["pref"], _abi.PREC_MIXED)
        while pending:
            drain(50)
    st = srv.stats()
    srv.close()
    wall = t_last - t0
    ok = [results[k]["status"] == 0 for k in sorted(results)]
    conv = [results[k]["status"] == 0 and results[k]["converged"] == 1 for k in sorted(results)]
    diverged = [results[k]["status"] == -5 for k in sorted(results)]
    lat = np.array([results[k]["total_ms"] for k in sorted(results) if conv[k]] or [np.nan])
    # parity sample: the smallest cases re-run alone
    check = []
    order = sorted([k for k in range(len(stream)) if conv[k]], key=lambda k: stream[k]["mesh"].ncells)[: a.serve_check]
    for k in order:
        c, r = stream[k], results[k]
        row = {"case": f"{c['kind']} N={c['N']} Re={c['Re']:.0f}", "iterations": r["iterations"]}
        for prec, name in ((_abi.PREC_MIXED, "alone_mixed"), (_abi.PREC_FP64, "alone_fp64")):
            case, keep = X.make_case(c["model"], c["config"], c["pref"], prec)
            s = X.Solver(c["mesh"], renumber=_abi.RENUMBER_COLOR)
            s.setup(case)
            s.set_tolerance(1e-6)
            U0, p0 = cases.fields(c["model"])
            for f, v in ((_abi.FIELD_UX, U0[0]), (_abi.FIELD_UY, U0[1]), (_abi.FIELD_UZ, U0[2]), (_abi.FIELD_P, p0)):
                s.set_field(f, v)
            out = s.run(a.serve_maxit, want_krylov=False)
            U = np.stack([s.get_field(_abi.FIELD_UX), s.get_field(_abi.FIELD_UY)])
            s.close()
            d = float(max(np.linalg.norm(U[i] - r["U"][i]) / max(np.linalg.norm(U[i]), 1e-300) for i in range(2)))
            row[name] = {"iterations": out["done"], "U_rel_l2": d}
        check.append(row)
    seq = serve_one_at_a_time(a, stream, results) if a.serve_seq > 0 else None
    value = len(results) / wall
    cit = st["cell_iterations"] / wall
    line = {
        "metric": "serving cases/s", "value": value, "unit": "cases/s", "n_gpus": 1,
        "steps": len(stream), "warmup": 0, "ms_per_step": 1000.0 * wall / max(len(results), 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
        "data": "synthetic cases from the seeded serving generator (numpy default_rng(12345))",
        "config": {"workload": f"{len(stream)} cavity/BFS cases, Poisson {a.serve_rate}/s, N in [40,{a.serve_nmax}], "
                               f"Re U(50,1000), stop at residuals <= 1e-6 (cap {a.serve_maxit})",
                   "slots": a.slots, "precision": "mixed", "launch": "one hardware cluster per case"},
        "time_to_converged_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                                 "max": float(np.max(lat)), "over": "converged cases, submit to result"},
        "finished": len(results), "converged": int(sum(conv)), "capped": int(sum(ok) - sum(conv)),
        "diverged": int(sum(diverged)), "failed_other": int(st["failed"] - sum(diverged)),
        "note": "value = finished cases (converged, capped or diverged) / wall time; diverged = non-finite "
                "Krylov norms, stopped early (the reference SIMPLE diverges on BFS above Re ~100-150)",
        "cell_iters_per_s": cit, "wall_s": wall,
        "one_at_a_time": seq,
        "vs_one_at_a_time": None if not seq else {
            "cases_per_s": value / seq["cases_per_s"], "cell_iters_per_s": cit / seq["cell_iters_per_s"],
            "note": "cases/s of the whole stream against an evenly spaced sample of it run one at a time; "
                    "cell-iters/s normalises the work of the two samples"},
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
    mesh, model, config, pref, desc = build_case(a.config, a.size)
    N = mesh.ncells
    workload = f"{a.config}_{N}_{a.precision}_simple"

    if a.impl == "reference":
        if rank != 0:
            return
        steps = a.steps
        rate, its, dt = cpu_oracle_rate(mesh, model, config, pref, seconds=min(120.0, max(5.0, a.cpu_seconds)))
        line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": a.gpus,
                "steps": its, "warmup": 0, "ms_per_step": 1000 * dt / its, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic mesh from the seeded generator (reference UNV construction rules)",
                "config": {"workload": desc, "cells": N, "renumber": "none (reference order)"},
                "cpu_baseline": {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
                                 "sample": f"first {its} SIMPLE iterations of the case ({dt:.1f} s), "
                                           f"CPU: {cpu_model()}"},
                "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    dist = init_ranks(world, local)
    import xcal as X
    from xcal import _abi, cases

    renum = {"color": _abi.RENUMBER_COLOR, "rcm": _abi.RENUMBER_RCM, "none": _abi.RENUMBER_NONE}[a.renumber]
    prec = _abi.PREC_MIXED if a.precision == "mixed" else _abi.PREC_FP64
    case, keep = X.make_case(model, config, pref, prec)
    s = X.Solver(mesh, device=local if world > 1 else 0, renumber=renum)
    s.setup(case)
    U0, p0 = cases.fields(model)
    dev = torch.device("cuda", local if world > 1 else 0)
    flush = None if a.no_flush else torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    turb = [(_abi.FIELD_K, model.turbulence.k.values.copy()), (_abi.FIELD_OMEGA, model.turbulence.omega.values.copy()),
            (_abi.FIELD_NUT, model.turbulence.nut.values.copy())] if X.isturbulent(model) else []

    def reset():
        for f, v in ((_abi.FIELD_UX, U0[0]), (_abi.FIELD_UY, U0[1]), (_abi.FIELD_UZ, U0[2]), (_abi.FIELD_P, p0)):
            s.set_field(f, v)
        for f, v in turb:
            s.set_field(f, v)

    def do_flush():
        if flush is not None:
            flush.fill_(1.0)
            torch.cuda.synchronize(dev)

    # warm-up (untimed), then restart the case from its initial fields
    reset()
    for _ in range(max(a.warmup, 0)):
        s.run(1, want_krylov=False)
    reset()
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ms = []
    kry = []
    gpu_index = local if world > 1 else int(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0] or 0)
    with ClockSampler(gpu_index) as clk:
        for k in range(a.steps):
            do_flush()
            out = s.run(1)
            ms.append(s.last_ms())
            kry.append(out["krylov"][0])
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    total_ms = max_over_ranks(float(sum(ms)), dist, dev)
    value = job_throughput(world, N * a.steps, total_ms / 1000.0)
    kry = np.array(kry)
    # roofline of the (single) device program kernel
    ns = 3 if mesh.dim == 3 else 2
    sk = 4 if a.precision == "mixed" else 8
    bytes_per_step = np.array([algorithmic_bytes(mesh, kr, ns, sk) for kr in kry], dtype=np.float64)
    achieved_gbs = float(bytes_per_step.sum() / (np.array(ms).sum() / 1000.0) / 1e9)
    peak, peak_kind = load_peaks()

    # end to end through the public API with host buffers
    e2e_steps = a.e2e_steps or min(a.steps, 100)
    reset()
    Uh = [U0[0].copy(), U0[1].copy()]
    ph = p0.copy()
    e2e_t = 0.0
    for k in range(e2e_steps):
        do_flush()
        t0 = time.perf_counter()
        s.set_field(_abi.FIELD_UX, Uh[0]); s.set_field(_abi.FIELD_UY, Uh[1]); s.set_field(_abi.FIELD_P, ph)
        out = s.run(1, want_krylov=False)
        Uh[0] = s.get_field(_abi.FIELD_UX); Uh[1] = s.get_field(_abi.FIELD_UY); ph = s.get_field(_abi.FIELD_P)
        e2e_t += time.perf_counter() - t0
    e2e_value = job_throughput(world, N * e2e_steps, max_over_ranks(e2e_t, dist, dev))
    h2d = 3 * N * 8
    d2h = 3 * N * 8 + 4 * 8 + 5 * 4
    s.close()

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        rate, its, dt = cpu_oracle_rate(mesh, model, config, pref, a.cpu_seconds)
        cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"CPU oracle, first {its} SIMPLE iterations of the same case ({dt:.1f} s), "
                         f"1 thread, {cpu_model()}"}
    clocks = clk.summary()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": total_ms / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if a.precision == "fp64" else "f64+f32",
        "data": "synthetic mesh from the seeded generator (reference UNV construction rules)",
        "config": {"workload": desc, "cells": N, "renumber": a.renumber, "precision": a.precision,
                   "step": "one SIMPLE iteration from zero initial fields",
                   "l2": "flushed between steps (256 MiB write)" if flush is not None else "not flushed",
                   "krylov_mean": {"U": float(kry[:, 0].mean()), "p": float(kry[:, 3].mean())},
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                     "frac": achieved_gbs / peak, "peak_kind": peak_kind,
                     "traffic": load_traffic(workload),
                     "kernel": "xcal_program_kernel (persistent SIMPLE iteration)"},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps},
        "gpu_launches": a.steps,
        "clocks": clocks,
        "impl": "xcal",
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
