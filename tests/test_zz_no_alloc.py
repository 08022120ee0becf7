"""GPU test of tsu_cfl_dt_noalloc, the CFL-step entry point that allocates
no device memory (for callers that cannot let a library call cudaMalloc:
frameworks that own all device memory through their own pool, services that
forbid allocation after start-up).

It is called through the C ABI on a state that the ordinary solver holds on
the device, twice in a row, and each result must equal the step the existing
entry points compute for the same state (tsu_reset for the initial state,
the end-of-step reduction of tsu_step for the next one) -- value for value,
the bar of the FP64 tests.  The output double is device memory that the test
owns.  This file is collected last on purpose, and passes alone too."""
import ctypes as C

import numpy as np
import pytest

import tsuner_b200 as T
from tsuner_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _noalloc_dt(s, p, out_ptr):
    ptr, pitch, plane, eb = s.device_state()
    assert eb == 8
    h = C.c_void_p(ptr)
    qx = C.c_void_p(ptr + plane * 8)
    qy = C.c_void_p(ptr + 2 * plane * 8)
    return T.lib().tsu_cfl_dt_noalloc(h, qx, qy, pitch, C.byref(p), C.c_void_p(out_ptr), None)


def test_noalloc_dt_matches_solver_on_two_calls():
    torch = pytest.importorskip("torch")
    w = W.nwave_shelf(600, 400, 20.0, slr=0.5, amp=2.0, period=300.0, t_series=400.0)
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    s = T.solver_for(w)
    try:
        t0, dt0, _ = s.time()  # dt computed by tsu_reset
        assert _noalloc_dt(s, w.p, out.data_ptr()) == 0
        s.step(30)
        t1, dt1, n1 = s.time()  # next dt computed by the last stage of step 30
        assert n1 == 30
        assert _noalloc_dt(s, w.p, out.data_ptr() + 8) == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
    finally:
        s.close()
    assert got[0] == dt0, (got[0], dt0)
    assert got[1] == dt1, (got[1], dt1)
    assert dt0 != dt1


def test_noalloc_dt_small_grid_exact_minimum():
    """At most 4096 cells the reference keeps the FP64 minimum (no float
    rounding): the entry point must agree with tsu_reset there too."""
    torch = pytest.importorskip("torch")
    w = W.hump(40, 24, 10.0, sigma=60.0)
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda:0")
    s = T.solver_for(w)
    try:
        _, dt0, _ = s.time()
        assert _noalloc_dt(s, w.p, out.data_ptr()) == 0
        assert _noalloc_dt(s, w.p, out.data_ptr() + 8) == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
    finally:
        s.close()
    assert got[0] == dt0 and got[1] == dt0, (got, dt0)
    assert float(np.float32(dt0)) != dt0  # the unrounded FP64 minimum


def test_noalloc_rejects_grids_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    w = W.hump(64, 48, 10.0)
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    s = T.solver_for(w)
    try:
        big = T.make_params(4096, 2048, 10.0, 10.0)  # 32768 CTAs > 16384
        ptr, pitch, plane, _ = s.device_state()
        rc = T.lib().tsu_cfl_dt_noalloc(C.c_void_p(ptr), C.c_void_p(ptr), C.c_void_p(ptr), 4096, C.byref(big),
                                        C.c_void_p(out.data_ptr()), None)
        assert rc == T.abi.TSU_ERR_INVALID
        assert b"partial minima" in T.lib().tsu_last_error()
    finally:
        s.close()
    assert np.isfinite(float(out.cpu()[0]))
