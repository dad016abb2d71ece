"""Device-side failure detection, the per-phase timers and the autotuner.

* The grid barrier's bounded wait: with XCAL_BARRIER_EXTRA=1 every wait
  expects one arrival more than the launch has CTAs, so it can only end by its
  wall-clock limit (XCAL_BARRIER_TIMEOUT_US, 1 ms here).  The run must come back
  with XCAL_ERR_TIMEOUT, without a device fault, and the same context must then
  run the case correctly (bitwise equal to a fresh context).
* XCAL_FLAG_PHASE_TIMERS: the number of phases charged to each class matches
  the run's own Krylov iteration counts, and every class that ran has cycles.
"""
import numpy as np
import pytest

import xcal as X
from xcal import _abi, cases

pytestmark = pytest.mark.gpu


def _solver(mesh, model, config, pref, flags=0):
    case, keep = X.make_case(model, config, pref)
    s = X.Solver(mesh, renumber=_abi.RENUMBER_COLOR, flags=flags)
    s.setup(case)
    U, p = cases.fields(model)
    for f, v in ((_abi.FIELD_UX, U[0]), (_abi.FIELD_UY, U[1]), (_abi.FIELD_UZ, U[2]), (_abi.FIELD_P, p)):
        s.set_field(f, v)
    return s, keep


def test_grid_barrier_wait_times_out_and_context_recovers(monkeypatch):
    mesh, model, config, pref = cases.cavity2d(20, iterations=10)
    monkeypatch.setenv("XCAL_SYNC", "grid")
    s, keep = _solver(mesh, model, config, pref)
    try:
        monkeypatch.setenv("XCAL_BARRIER_EXTRA", "1")
        monkeypatch.setenv("XCAL_BARRIER_TIMEOUT_US", "1000")
        with pytest.raises(_abi.XcalError, match="XCAL_ERR_TIMEOUT"):
            s.run(10)
        assert s.last_ms() < 1000.0, "the run ended by the 1 ms wait limit"
        monkeypatch.delenv("XCAL_BARRIER_EXTRA")
        monkeypatch.delenv("XCAL_BARRIER_TIMEOUT_US")
        U, p = cases.fields(model)   # the aborted run may have touched the fields: start again
        for f, v in ((_abi.FIELD_UX, U[0]), (_abi.FIELD_UY, U[1]), (_abi.FIELD_UZ, U[2]), (_abi.FIELD_P, p)):
            s.set_field(f, v)
        got = s.run(10)
        Ug = np.stack([s.get_field(_abi.FIELD_UX), s.get_field(_abi.FIELD_UY)])
    finally:
        s.close()
    fresh, keep2 = _solver(mesh, model, config, pref)
    try:
        ref = fresh.run(10)
        Ur = np.stack([fresh.get_field(_abi.FIELD_UX), fresh.get_field(_abi.FIELD_UY)])
    finally:
        fresh.close()
    assert got["done"] == ref["done"] == 10
    assert np.array_equal(Ug, Ur)
    assert np.array_equal(np.nan_to_num(got["R_p"]), np.nan_to_num(ref["R_p"]))


@pytest.mark.parametrize("sync", ["cluster", "grid"])
def test_phase_timers_count_the_run(sync, monkeypatch):
    monkeypatch.setenv("XCAL_SYNC", sync)
    mesh, model, config, pref = cases.bfs(6, iterations=8)
    s, keep = _solver(mesh, model, config, pref, flags=_abi.FLAG_PHASE_TIMERS)
    try:
        out = s.run(8)
        ph = s.last_phases()
        nfl = int(s.csr()[4][0])
    finally:
        s.close()
    kry = out["krylov"][: out["done"]]
    itU = kry[:, :2].max(axis=1).sum()
    itP = kry[:, 3].sum()
    n = out["done"]
    # BiCGSTAB: 2 SpMV phases per iteration, CG: 1 (a CG stopped by zero
    # curvature runs one SpMV phase without counting an iteration)
    assert 2 * itU + itP <= ph["krylov_spmv"][1] <= 2 * itU + itP + n
    assert ph["momentum_assembly"][1] == n and ph["pressure_assembly"][1] == n
    assert ph["residual"][1] == 2 * n
    assert nfl == 2
    for k in ("momentum_assembly", "pressure_assembly", "precon_setup", "krylov_spmv", "krylov_precon",
              "residual", "face", "gradient", "update"):
        assert ph[k][0] > 0 and ph[k][1] > 0, k
    assert ph["turbulence"] == (0.0, 0)


def test_autotune_keeps_results_and_picks_a_form():
    """xcal_autotune times the launch forms on the case, restores its fields
    and keeps the fastest; the tuned run equals an untuned one bit for bit,
    and the tuned form is no slower than the default it was timed against."""
    mesh, model, config, pref = cases.bfs(9, iterations=12)
    s, keep = _solver(mesh, model, config, pref)
    try:
        choice = s.autotune(iterations=3)
        assert choice["candidates"] >= 2 and choice["ctas"] >= 1 and choice["ctas_per_sm"] in (2, 4)
        assert choice["ms_per_iteration"] <= choice["ms_default"]
        tuned = s.run(12)
        Ut = np.stack([s.get_field(_abi.FIELD_UX), s.get_field(_abi.FIELD_UY)])
    finally:
        s.close()
    ref_s, keep2 = _solver(mesh, model, config, pref)
    try:
        ref = ref_s.run(12)
        Ur = np.stack([ref_s.get_field(_abi.FIELD_UX), ref_s.get_field(_abi.FIELD_UY)])
    finally:
        ref_s.close()
    assert tuned["done"] == ref["done"] == 12
    assert np.array_equal(Ut, Ur)
    assert np.array_equal(np.nan_to_num(tuned["R_p"]), np.nan_to_num(ref["R_p"]))
