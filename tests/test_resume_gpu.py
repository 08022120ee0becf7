"""GPU: checkpoint and resume (tsu_resume).  A run interrupted after k steps
and continued from its checkpoint (state, extrema, t and step count read back
through the C ABI, loaded into a new solver) must equal the uninterrupted run:
value for value in the FP64 form (order 2 with a boundary series, order 1
with its ping-pong buffers), within float round-off in the FP32 form."""
import numpy as np
import pytest

import tsuner_b200 as T
from tsuner_b200 import workloads as W
from tsuner_b200.abi import TSU_ERR_INVALID, make_switches

pytestmark = pytest.mark.gpu


def fresh(w, sw):
    s = T.Solver(w.p, sw)
    s.set_state(w.V)
    s.set_mask(w.mask)
    if sw.read_files:
        s.set_boundary_series(w.CC, w.tCC)
    s.reset()
    return s


def checkpoint_and_continue(w, sw, k, n):
    s = fresh(w, sw)
    s.step(k)
    V, ext, (t, _, steps) = s.state(), s.extrema(), s.time()
    s.close()
    s = T.Solver(w.p, sw)
    try:
        s.set_state(V)
        s.set_mask(w.mask)
        if sw.read_files:
            s.set_boundary_series(w.CC, w.tCC)
        s.reset()
        s.resume(t, steps, ext)
        s.step(n - k)
        return s.state(), s.extrema(), s.time()
    finally:
        s.close()


@pytest.mark.parametrize("order", [2, 1])
def test_fp64_resume_continues_value_for_value(order):
    w = W.nwave_shelf(160, 96, 20.0, slr=0.5, amp=2.0, period=200.0, t_series=300.0)
    sw = make_switches(order=order, wbc=w.sw.wbc, read_files=1, precision=0, eta0=w.sw.eta0)
    s = fresh(w, sw)
    s.step(31)
    V, ext, tm = s.state(), s.extrema(), s.time()
    s.close()
    V2, ext2, tm2 = checkpoint_and_continue(w, sw, 13, 31)
    assert tm2 == tm
    assert np.array_equal(V2, V)
    for a, b in zip(ext2, ext):
        assert np.array_equal(a, b)


def test_fp32_resume_continues_within_round_off():
    w = W.nwave_shelf(160, 96, 20.0, slr=0.5, amp=2.0, period=200.0, t_series=300.0)
    sw = make_switches(order=2, wbc=w.sw.wbc, read_files=1, precision=1, eta0=w.sw.eta0)
    s = fresh(w, sw)
    s.step(31)
    V, ext, (t, _, n) = s.state(), s.extrema(), s.time()
    s.close()
    V2, ext2, (t2, _, n2) = checkpoint_and_continue(w, sw, 13, 31)
    assert n2 == n and abs(t2 - t) <= 1e-6 * t
    assert np.abs(V2[0] - V[0]).max() <= 1e-4
    assert np.abs(ext2[0] - ext[0]).max() <= 1e-4


def test_resume_needs_a_reset_state_and_valid_arguments():
    w = W.hump(40, 30, 10.0, sigma=60.0)
    s = T.Solver(w.p, w.sw)
    try:
        s.set_state(w.V)
        assert T.lib().tsu_resume(s._h, 1.0, 3, None, None, None) == TSU_ERR_INVALID  # before tsu_reset
        s.reset()
        assert T.lib().tsu_resume(s._h, -1.0, 3, None, None, None) == TSU_ERR_INVALID
        assert T.lib().tsu_resume(s._h, 1.0, -3, None, None, None) == TSU_ERR_INVALID
        s.resume(2.5, 7)  # extrema keep their fresh fill
        t, _, n = s.time()
        assert t == 2.5 and n == 7
        s.step(1)
        assert s.time()[2] == 8 and s.time()[0] > 2.5
    finally:
        s.close()
