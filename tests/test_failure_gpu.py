"""GPU: the error paths of the kernels, exercised without a GPU fault.

* Expired waits.  Every wait of a stage kernel or a corrector convolution on
  its own TMA copies / MMAs is bounded; tsu_set_wait_limit_ns lowers that
  bound to a few nanoseconds so that the waits run out while the copies are
  still in flight (nothing else changes: the copies are ordinary and land
  microseconds later).  The kernels must record the error (TSU_ERR_CUDA from
  tsu_sync / tsu_corr_status), drain their copies and MMAs, free their
  tensor memory and return; with the normal limit the same solver, after
  tsu_reset, must step to the same values as a fresh one, and a convolution
  must again equal its PyTorch FP32 reference.
* Non-finite states.  A NaN planted in the HOST state before tsu_set_state is
  reported by tsu_reset; a NaN written into the device state between steps
  (through the library's own copy call) is reported after the next step, by
  tsu_sync and tsu_run_until, for both forms and for an ensemble member.
"""
import ctypes as C

import numpy as np
import pytest

import tsuner_b200 as T
from tsuner_b200 import workloads as W
from tsuner_b200.abi import TSU_ERR_CUDA, TSU_ERR_NONFINITE, make_switches

pytestmark = pytest.mark.gpu


def sw_of(w, precision):
    return make_switches(order=2, wbc=w.sw.wbc, read_files=w.sw.read_files, precision=precision, eta0=w.sw.eta0)


def loaded(w, precision):
    s = T.Solver(w.p, sw_of(w, precision))
    s.set_state(w.V)
    s.set_mask(w.mask)
    if w.sw.read_files:
        s.set_boundary_series(w.CC, w.tCC)
    s.reset()
    return s


@pytest.fixture
def short_waits():
    """Lowers the wait limit for the test body; always restores the default."""
    L = T.lib()
    L.tsu_set_wait_limit_ns.argtypes = [C.c_ulonglong]
    L.tsu_set_wait_limit_ns.restype = C.c_int

    def set_limit(ns):
        assert L.tsu_set_wait_limit_ns(ns) == 0

    yield set_limit
    assert L.tsu_set_wait_limit_ns(0) == 0


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_expired_tile_wait_is_reported_and_the_solver_recovers(precision, short_waits):
    # 512 x 384 cells: most tiles are interior tiles, which stage by TMA
    w = W.nwave_shelf(512, 384, 10.0, slr=0.5, amp=2.0, period=300.0, t_series=400.0)
    ref = loaded(w, precision)
    ref.step(20)
    V_ref = ref.state()
    ref.close()

    s = loaded(w, precision)
    s.step(3)
    s.sync()
    short_waits(1)
    assert T.lib().tsu_step(s._h, 2) == 0  # enqueues; the error shows at the sync
    rc = T.lib().tsu_sync(s._h)
    assert rc == TSU_ERR_CUDA, rc
    assert b"expired" in T.lib().tsu_last_error()
    assert T.lib().tsu_step(s._h, 1) == TSU_ERR_CUDA  # refuses to step until reset
    short_waits(0)
    s.set_state(w.V)
    s.reset()
    s.step(20)
    V = s.state()
    t = s.time()
    s.close()
    assert t[2] == 20
    assert np.array_equal(V, V_ref)


def test_expired_ensemble_wait_is_reported(short_waits):
    ws = W.ensemble(nmembers=3, lo=200, hi=300, seed=9, dx=20.0, t_series=200.0)
    e = T.Ensemble([m.p for m in ws], [m.sw for m in ws])
    try:
        e.load(ws)
        e.reset()
        e.step(2)
        e.sync()
        short_waits(1)
        assert T.lib().tsu_ens_step(e._h, 2) == 0
        assert T.lib().tsu_ens_sync(e._h) == TSU_ERR_CUDA
        short_waits(0)
        e.load(ws)
        e.reset()
        e.step(5)
        e.sync()
        assert all(np.isfinite(m.state()).all() for m in e.members)
    finally:
        e.close()


def test_expired_convolution_waits_are_reported_and_clear(short_waits):
    torch = pytest.importorskip("torch")
    F = torch.nn.functional
    g = torch.Generator().manual_seed(3)
    n, h, wd = 2, 96, 80
    Xt = torch.randn(n, 32, h, wd, generator=g).to(torch.bfloat16)
    Wt = (torch.randn(32, 32, 3, 3, generator=g) * 0.1).to(torch.bfloat16)
    dev = torch.device("cuda:0")
    X = Xt.permute(0, 2, 3, 1).contiguous().to(dev)
    Wk = Wt.permute(0, 2, 3, 1).reshape(32, 9, 32).contiguous().to(dev)
    dZ = torch.randn(n, h, wd, 32, generator=g).to(torch.bfloat16).to(dev)
    Y = torch.zeros((n, h, wd, 32), device=dev, dtype=torch.float32)
    dW = torch.zeros((32, 288), device=dev, dtype=torch.float32)
    db = torch.zeros(32, device=dev, dtype=torch.float32)
    L = T.lib()

    def fwd():
        return L.tsu_corr_conv3x3(C.c_void_p(X.data_ptr()), n, h, wd, C.c_void_p(Wk.data_ptr()), None, 0, None,
                                  None, C.c_void_p(Y.data_ptr()), None)

    def wgrad():
        return L.tsu_corr_conv3x3_wgrad(C.c_void_p(X.data_ptr()), C.c_void_p(dZ.data_ptr()), n, h, wd,
                                        C.c_void_p(dW.data_ptr()), C.c_void_p(db.data_ptr()), None)

    torch.cuda.synchronize()
    short_waits(1)
    assert fwd() == 0
    assert L.tsu_corr_status() == TSU_ERR_CUDA
    assert wgrad() == 0
    assert L.tsu_corr_status() == TSU_ERR_CUDA
    short_waits(0)
    Y.zero_()
    dW.zero_()
    db.zero_()
    assert fwd() == 0 and wgrad() == 0
    assert L.tsu_corr_status() == 0
    ref = F.conv2d(Xt.float(), Wt.float(), padding=1).permute(0, 2, 3, 1).to(dev)
    assert torch.allclose(Y, ref, rtol=1e-4, atol=1e-4 * float(ref.abs().max()))
    dZn = dZ.float().permute(0, 3, 1, 2).cpu()
    ref_dW = torch.nn.grad.conv2d_weight(Xt.float(), (32, 32, 3, 3), dZn, padding=1)
    got = dW.cpu().reshape(32, 3, 3, 32).permute(0, 3, 1, 2)
    assert torch.allclose(got, ref_dW, rtol=1e-4, atol=1e-4 * float(ref_dW.abs().max()))
    assert torch.allclose(db.cpu(), dZn.sum(dim=(0, 2, 3)), rtol=1e-4, atol=1e-3)


@pytest.mark.parametrize("precision,plane", [(0, 0), (0, 1), (1, 1), (1, 3)], ids=["fp64_h", "fp64_qx", "fp32_qx",
                                                                                    "fp32_H"])
def test_nan_in_uploaded_host_state_is_reported(precision, plane):
    w = W.hump(70, 50, 10.0, sigma=80.0)
    w.V[plane, 20, 30] = np.nan
    s = T.Solver(w.p, sw_of(w, precision))
    try:
        s.set_state(w.V)
        with pytest.raises(T.TsunerError) as ei:
            s.reset()
        assert ei.value.code == TSU_ERR_NONFINITE
        assert b"NaN" in T.lib().tsu_last_error()
        # a finite state clears it
        w2 = W.hump(70, 50, 10.0, sigma=80.0)
        s.set_state(w2.V)
        s.reset()
        s.step(3)
        s.sync()
    finally:
        s.close()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_nan_appearing_between_steps_is_reported(precision):
    w = W.hump(70, 50, 10.0, sigma=80.0)
    s = loaded(w, precision)
    try:
        s.step(2)
        s.sync()
        ptr, pitch, plane, eb = s.device_state()
        # one NaN into the qx plane (plane 1 of FP64, plane 2 of FP32), cell (row 25, column 35)
        f = 1 if precision == 0 else 2
        off = (f * plane + 25 * pitch + 35) * eb
        bad = np.array([np.nan], np.float64 if eb == 8 else np.float32)
        assert T.lib().tsu_copy_bytes_to_device(0, C.c_void_p(ptr + off), bad.ctypes.data_as(C.c_void_p), eb) == 0
        with pytest.raises(T.TsunerError) as ei:  # run_until checks after each chunk of steps
            s.run_until(1e9, 4)
        assert ei.value.code == TSU_ERR_NONFINITE
        with pytest.raises(T.TsunerError) as ei:  # the device's status word stays set
            s.sync()
        assert ei.value.code == TSU_ERR_NONFINITE
        assert T.lib().tsu_step(s._h, 1) == TSU_ERR_NONFINITE  # no stepping until reset
        assert b"tsu_reset" in T.lib().tsu_last_error()
    finally:
        s.close()


def test_nan_in_one_ensemble_member_is_reported():
    ws = W.ensemble(nmembers=2, lo=60, hi=90, seed=5, dx=20.0, t_series=100.0)
    e = T.Ensemble([m.p for m in ws], [m.sw for m in ws])
    try:
        e.load(ws)
        e.reset()
        e.step(2)
        e.sync()
        m = e.members[1]
        ptr, pitch, plane, eb = m.device_state()
        bad = np.array([np.nan], np.float32)
        assert T.lib().tsu_copy_bytes_to_device(0, C.c_void_p(ptr + (2 * plane + 10 * pitch + 10) * eb),
                                                bad.ctypes.data_as(C.c_void_p), eb) == 0
        e.step(1)
        assert T.lib().tsu_ens_sync(e._h) == TSU_ERR_NONFINITE
    finally:
        e.close()
