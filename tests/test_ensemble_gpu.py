"""GPU: the batched ensemble (one persistent launch per RK stage over the
tiles of all members) against the same members stepped one by one with the
single-grid FP32 kernels.  The per-cell arithmetic does not depend on how
tiles are scheduled, so every member's state, time and dt must be equal value
for value, for every tile shape and schedule, and after the autotuner (which
must restore the members' states)."""
import numpy as np
import pytest

import tsuner_b200 as T
from tsuner_b200 import workloads as W

pytestmark = pytest.mark.gpu

STEPS = 40


def small_ensemble():
    ws = W.ensemble(nmembers=6, lo=40, hi=260, seed=11, dx=20.0, t_series=200.0)
    ws[2].sw.read_files = 0  # one member with plain walls
    return ws


def run_alone(w, steps):
    s = T.Solver(w.p, w.sw)
    s.set_state(w.V)
    s.set_mask(w.mask)
    if w.sw.read_files:
        s.set_boundary_series(w.CC, w.tCC)
    s.reset()
    s.step(steps)
    out = (s.state(), s.time())
    s.close()
    return out


@pytest.fixture(scope="module")
def reference_runs():
    ws = small_ensemble()
    return ws, [run_alone(w, STEPS) for w in ws]


def make_ens(ws):
    e = T.Ensemble([w.p for w in ws], [w.sw for w in ws])
    e.load(ws)
    e.reset()
    return e


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
@pytest.mark.parametrize("schedule", ["static", "dynamic", "one_per_tile"])
def test_ensemble_equals_members_alone(reference_runs, variant, schedule):
    ws, ref = reference_runs
    e = make_ens(ws)
    if schedule == "one_per_tile":
        e.set_config(variant, 0, 1 << 30)
    else:
        e.set_config(variant, 1 if schedule == "dynamic" else 0, 0)
    e.step(STEPS)
    e.sync()
    for k, s in enumerate(e.members):
        V = s.state()
        t = s.time()
        assert np.array_equal(V, ref[k][0]), (k, np.abs(V - ref[k][0]).max())
        assert t[0] == ref[k][1][0] and t[1] == ref[k][1][1] and t[2] == STEPS
    dts = {round(s.time()[1], 12) for s in e.members}
    assert len(dts) > 1  # members advance with their own dt
    e.close()


def test_autotune_restores_state_and_picks_a_config(reference_runs):
    ws, ref = reference_runs
    e = make_ens(ws)
    report = e.autotune(steps=2)
    assert "ms/step" in report and len(report.splitlines()) >= 8
    cfg = e.config()
    assert cfg["ntiles"] > 0 and cfg["ctas"] > 0
    e.step(STEPS)
    e.sync()
    for k, s in enumerate(e.members):
        assert np.array_equal(s.state(), ref[k][0])
        assert s.time()[2] == STEPS
    e.close()


def test_run_until_stops_each_member_at_its_end_time(reference_runs):
    """tsu_ens_run_until: every member reaches t_end with its own step count
    and then skips its tiles; each member's state equals the same member run
    alone with tsu_run_until."""
    ws, _ = reference_runs
    t_end = 6.0
    alone = []
    for w in ws:
        s = T.Solver(w.p, w.sw)
        s.set_state(w.V)
        s.set_mask(w.mask)
        if w.sw.read_files:
            s.set_boundary_series(w.CC, w.tCC)
        s.reset()
        s.run_until(t_end)
        alone.append((s.state(), s.time()))
        s.close()
    e = make_ens(ws)
    e.run_until(t_end)
    e.sync()
    for k, s in enumerate(e.members):
        t, dt, n = s.time()
        assert t >= t_end
        assert (t, dt, n) == alone[k][1]
        assert np.array_equal(s.state(), alone[k][0])
    steps = {s.time()[2] for s in e.members}
    assert len(steps) > 1  # members needed different numbers of steps
    e.step(1)  # run_until restores the open end time
    e.sync()
    assert all(s.time()[2] == alone[k][1][2] + 1 for k, s in enumerate(e.members))
    e.close()


def test_members_follow_the_fp64_plain_form(reference_runs):
    """Each member of the ensemble against the same member in the FP64 plain
    form (the reference's arithmetic) after the same simulated time: depth
    within the FP32 form's run-up bound (2e-3 m, tests/test_fp32_gpu.py) and
    the water volume within 1e-6 relative."""
    from tsuner_b200.abi import make_switches
    ws, _ = reference_runs
    t_end = 8.0
    e = make_ens(ws)
    e.run_until(t_end)
    e.sync()
    try:
        for k, w in enumerate(ws):
            m = e.members[k]
            V32, (t32, _, _) = m.state(), m.time()
            sw64 = make_switches(order=w.sw.order, wbc=w.sw.wbc, read_files=w.sw.read_files, precision=0,
                                 eta0=w.sw.eta0)
            s = T.Solver(w.p, sw64)
            try:
                s.set_state(w.V)
                s.set_mask(w.mask)
                if w.sw.read_files:
                    s.set_boundary_series(w.CC, w.tCC)
                s.reset()
                s.run_until(t_end)
                V64, (t64, _, _) = s.state(), s.time()
            finally:
                s.close()
            assert abs(t32 - t64) <= 1e-3 * t64
            linf = np.abs(V32[0] - V64[0]).max()
            assert linf <= 2e-3, (k, linf)
            m32, m64 = V32[0].sum(), V64[0].sum()
            assert abs(m32 - m64) <= 1e-6 * m64, (k, m32, m64)
    finally:
        e.close()
