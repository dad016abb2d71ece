"""Serving loop (xcal_serve_*): a stream of independent cases run concurrently
on one GPU inside one persistent launch, each case on a group of its CTAs.

A case's result inside the mix must equal its result run alone through the
plain path (one context, same precision, same stop tolerance): the device
program's arithmetic does not depend on the launch form, the number of CTAs
or other work on the GPU, so the comparison is bitwise (iteration count,
residual history end, fields).  Mixed-precision results are also compared
with the FP64 plain path (relative L2, reported)."""
import numpy as np
import pytest

import xcal as X
from xcal import _abi, cases
from parity_util import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-6
MAXIT = 3000


def _alone(c, precision, maxit=MAXIT):
    case, keep = X.make_case(c["model"], c["config"], c["pref"], precision)
    s = X.Solver(c["mesh"], renumber=_abi.RENUMBER_COLOR)
    try:
        s.setup(case)
        s.set_tolerance(TOL)
        U, p = cases.fields(c["model"])
        for f, v in ((_abi.FIELD_UX, U[0]), (_abi.FIELD_UY, U[1]), (_abi.FIELD_UZ, U[2]), (_abi.FIELD_P, p)):
            s.set_field(f, v)
        out = s.run(maxit, want_krylov=False)
        out["U"] = np.stack([s.get_field(_abi.FIELD_UX), s.get_field(_abi.FIELD_UY), s.get_field(_abi.FIELD_UZ)])
        out["p"] = s.get_field(_abi.FIELD_P)
    finally:
        s.close()
    return out


@pytest.mark.parametrize("precision", [_abi.PREC_FP64, _abi.PREC_MIXED], ids=["fp64", "mixed"])
def test_serve_matches_alone(precision):
    # Re <= 60: the reference SIMPLE (upwind, no Rhie-Chow, relax 0.7/0.3)
    # diverges on the coarse BFS meshes from about Re 125 (the CPU oracle
    # does the same), and those cases are covered by the divergence test.
    stream = cases.serving_stream(6, rate=1000.0, seed=7, nmin=16, nmax=48, re_max=60.0)
    srv = X.Server(slots=4, max_iterations=MAXIT, tolerance=TOL, precision=precision)
    try:
        tickets = [srv.submit(c["model"], c["config"], c["pref"]) for c in stream]
        results = [srv.poll(t, wait_ms=-1) for t in tickets]
        st = srv.stats()
    finally:
        srv.close()
    assert st["completed"] == len(stream) and st["failed"] == 0
    for c, r in zip(stream, results):
        assert r["status"] == 0
        a = _alone(c, precision)
        assert r["iterations"] == a["done"], (c["kind"], c["N"], r["iterations"], a["done"])
        assert r["converged"] == 1 and a["done"] < MAXIT
        last = a["done"] - 1
        assert r["residual"][0] == a["R_ux"][last] and r["residual"][3] == a["R_p"][last]
        assert np.array_equal(r["U"], a["U"]) and np.array_equal(r["p"], a["p"])
        if precision == _abi.PREC_MIXED:
            f = _alone(c, _abi.PREC_FP64)
            d = max(rel_l2(r["U"][0], f["U"][0]), rel_l2(r["U"][1], f["U"][1]))
            print(c["kind"], c["N"], round(c["Re"]), "mixed vs fp64 U rel L2", d, r["iterations"], f["done"])
            assert d <= 1e-3



def test_serve_concurrent_groups_repeatable():
    """Several multi-CTA cases in flight at once, repeated: every result equals
    the case run alone, bit for bit, in every repetition.  Groups of
    different cases share SMs, so a group's CTAs run at uneven speeds; a CTA
    that is still reading one reduction's partial sums while a faster CTA of
    its group writes the next reduction's must not see the new values (the
    partial sums are double-buffered for this)."""
    stream = cases.serving_stream(6, rate=1000.0, seed=7, nmin=16, nmax=48, re_max=60.0)
    alone = [_alone(c, _abi.PREC_FP64) for c in stream]
    for rep in range(3):
        srv = X.Server(slots=4, max_iterations=MAXIT, tolerance=TOL, precision=_abi.PREC_FP64, tiles_per_cta=1)
        try:
            tickets = [srv.submit(c["model"], c["config"], c["pref"]) for c in stream]
            results = [srv.poll(t, wait_ms=-1) for t in tickets]
        finally:
            srv.close()
        for k, (r, a) in enumerate(zip(results, alone)):
            assert r["status"] == 0, (rep, k, r["status"])
            assert r["iterations"] == a["done"], (rep, k, r["iterations"], a["done"])
            assert np.array_equal(r["U"], a["U"]) and np.array_equal(r["p"], a["p"]), (rep, k)

def test_serve_stats_and_errors():
    srv = X.Server(slots=2, max_iterations=50, tolerance=TOL)
    try:
        c = cases.serving_stream(1, seed=3, nmin=16, nmax=16, re_max=60.0)[0]
        t = srv.submit(c["model"], c["config"], c["pref"])
        r = srv.poll(t, wait_ms=-1)
        assert r["status"] == 0 and r["iterations"] <= 50
        with pytest.raises(_abi.XcalError):
            srv.poll(t)                  # a ticket is released once its result was read
        st = srv.stats()
        assert st["submitted"] == 1 and st["completed"] == 1 and st["queued"] == 0 and st["running"] == 0
        assert st["cell_iterations"] == c["mesh"].ncells * r["iterations"]
    finally:
        srv.close()


def test_serve_stops_a_diverged_case():
    """A case whose residuals become non-finite is stopped at that iteration
    (XCAL_FLAG_ABORT_ON_NAN on the serving contexts) and reported with status
    XCAL_ERR_NAN; the other cases are unaffected."""
    stream = cases.serving_stream(2, rate=1000.0, seed=11, nmin=16, nmax=24, re_max=60.0)
    bad = stream[0]
    bad["model"].p.values[3] = np.nan
    srv = X.Server(slots=2, max_iterations=500, tolerance=TOL)
    try:
        tb = srv.submit(bad["model"], bad["config"], bad["pref"])
        tg = srv.submit(stream[1]["model"], stream[1]["config"], stream[1]["pref"])
        rb = srv.poll(tb, wait_ms=-1)
        rg = srv.poll(tg, wait_ms=-1)
        st = srv.stats()
    finally:
        srv.close()
    assert rb["status"] == -5 and rb["iterations"] == 1
    assert rg["status"] == 0 and rg["converged"] == 1
    assert st["failed"] == 1 and st["completed"] == 1


@pytest.mark.parametrize("max_ctas", [1, 7, 64])
def test_serve_large_case_matches_alone(max_ctas):
    """A 14,400-cell case (57 tiles) run by groups of 1, 7 and 64 CTAs of the
    serving launch equals the case run alone (grid launch of the ordinary
    program) bit for bit."""
    mesh, model, config, pref = cases.cavity2d(120, iterations=1)
    c = dict(mesh=mesh, model=model, config=config, pref=pref)
    srv = X.Server(slots=1, max_iterations=400, tolerance=TOL, precision=_abi.PREC_FP64, tiles_per_cta=1,
                   max_ctas=max_ctas)
    try:
        r = srv.poll(srv.submit(model, config, pref), wait_ms=-1)
    finally:
        srv.close()
    a = _alone(c, _abi.PREC_FP64, maxit=400)
    assert r["status"] == 0 and r["iterations"] == a["done"]
    assert np.array_equal(r["U"], a["U"]) and np.array_equal(r["p"], a["p"])


def test_serve_admission_by_footprint():
    """With a device arena that holds about one case at a time, every case
    still runs (each waits for the previous one's memory) and the arena's
    peak use stays within it."""
    stream = cases.serving_stream(4, rate=1000.0, seed=5, nmin=40, nmax=40, re_max=60.0)
    srv = X.Server(slots=8, max_iterations=200, tolerance=TOL, precision=_abi.PREC_FP64,
                   device_bytes=6e6)
    try:
        tickets = [srv.submit(c["model"], c["config"], c["pref"]) for c in stream]
        results = [srv.poll(t, wait_ms=-1) for t in tickets]
        st = srv.stats()
    finally:
        srv.close()
    assert all(r["status"] == 0 for r in results), [r["status"] for r in results]
    assert st["device_bytes_peak"] <= st["device_bytes"] <= 6e6
    for c, r in zip(stream, results):
        a = _alone(c, _abi.PREC_FP64, maxit=200)
        assert r["iterations"] == a["done"] and np.array_equal(r["p"], a["p"])


def test_serve_rejects_a_case_of_another_dimension():
    srv = X.Server(slots=2, max_iterations=20, tolerance=TOL, precision=_abi.PREC_FP64, dim=2)
    try:
        mesh, model, config, pref = cases.cavity3d(6, iterations=1)
        r = srv.poll(srv.submit(model, config, pref), wait_ms=-1)
    finally:
        srv.close()
    assert r["status"] == -9   # XCAL_ERR_UNSUPPORTED
