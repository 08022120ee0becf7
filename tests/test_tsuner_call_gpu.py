"""GPU: the TSUNER() drop-in called directly through the C ABI, as the
reference's main_TSUNER.cxx:85-98 calls it, with a boundary series, a mask
with non-erodible cells and the shipped switches (Read_files = 1); and its
return codes (GPU/main_TSUNER.cu:20, main_TSUNER.cxx:91-98): 1 when the GPU
memory does not suffice, 2 when the output cannot be created, 3 for invalid
input.  The written file must equal the same run through the tsu_* API."""
import ctypes as C
import os

import numpy as np
import pytest

import tsuner_b200 as T
from tsuner_b200 import workloads as W
from tsuner_b200.abi import SimParams, TsuSwitches

pytestmark = pytest.mark.gpu


class Double2(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double)]


def bind():
    L = T.lib()
    dp = C.POINTER(C.c_double)
    fp = C.POINTER(C.c_float)
    L.TSUNER.argtypes = [dp, C.POINTER(Double2), dp, C.POINTER(C.c_int), SimParams, C.c_char_p, dp, dp, dp,
                         C.c_ulong, dp, fp, dp, C.c_int, dp, fp, C.c_int]
    L.TSUNER.restype = C.c_int
    L.tsu_set_default_switches.argtypes = [C.POINTER(TsuSwitches)]
    L.tsu_get_default_switches.argtypes = [C.POINTER(TsuSwitches)]
    return L


@pytest.fixture
def switches():
    """Sets the process-wide switches TSUNER() uses; restores them after."""
    L = bind()
    saved = TsuSwitches()
    assert L.tsu_get_default_switches(C.byref(saved)) == 0

    def set_sw(sw):
        assert L.tsu_set_default_switches(C.byref(sw)) == 0

    yield set_sw
    assert L.tsu_set_default_switches(C.byref(saved)) == 0


def dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def call_tsuner(w, prefix, mask=None, with_series=True, device=0):
    """TSUNER(h, (qx, qy), H, fixH, params, prefix, d, CC, tCC, timeCC, ...)."""
    L = bind()
    n = w.p.npx * w.p.npy
    h = np.ascontiguousarray(w.V[0].reshape(-1))
    H = np.ascontiguousarray(w.V[3].reshape(-1))
    q = (Double2 * n)()
    qa = np.frombuffer(q, np.float64).reshape(n, 2)
    qa[:, 0] = w.V[1].reshape(-1)
    qa[:, 1] = w.V[2].reshape(-1)
    m = np.ascontiguousarray((w.mask if mask is None else mask).reshape(-1), np.int32)
    CC = np.ascontiguousarray(w.CC, np.float64) if with_series else None
    tCC = np.ascontiguousarray(w.tCC, np.float64) if with_series else None
    tiempo = C.c_double(-1.0)
    rc = L.TSUNER(dptr(h), q, dptr(H), m.ctypes.data_as(C.POINTER(C.c_int)), w.p, prefix.encode(), None,
                  None if CC is None else dptr(CC), None if tCC is None else dptr(tCC),
                  0 if tCC is None else len(tCC), None, None, C.byref(tiempo), device, None, None, -1)
    return rc, tiempo.value


def shelf(total_time, save_time):
    w = W.nwave_shelf(96, 64, 20.0, slr=0.5, amp=3.0, period=200.0, t_series=300.0)
    w.p.total_time = total_time
    w.p.save_time = save_time
    assert w.sw.read_files == 1 and (w.mask == 0).any()
    return w


def test_tsuner_with_series_and_mask_matches_api_run(tmp_path, switches):
    from scipy.io import netcdf_file
    w = shelf(60.0, 20.0)
    switches(w.sw)
    prefix = str(tmp_path / "shelf")
    rc, tiempo = call_tsuner(w, prefix)
    assert rc == 0, T.lib().tsu_last_error()
    assert tiempo >= 0.0
    f = netcdf_file(prefix + ".nc", "r", mmap=False)
    try:
        t = f.variables["time"][:].copy()
        eta = f.variables["eta"][:].copy()
        ux = f.variables["ux"][:].copy()
        uy = f.variables["uy"][:].copy()
        hmax = f.variables["hmax"][:].copy()
        bmin = f.variables["bmin"][:].copy()
        eta_max = f.variables["eta_max"][:].copy()
    finally:
        f.close()
    assert t[0] == 0.0 and len(t) >= 4 and t[-1] >= 60.0  # frames at 0, 20, 40 and the final one
    def api_run(mask):
        s = T.Solver(w.p, w.sw)
        try:
            s.set_state(w.V)
            s.set_mask(mask)
            s.set_boundary_series(w.CC, w.tCC)
            s.reset()
            s.run_until(60.0)
            return s.state(), s.extrema(), s.time()
        finally:
            s.close()

    V, (hm, bm, em), (tt, _, _) = api_run(w.mask)
    eps = np.finfo(np.float64).eps
    assert tt == t[-1]
    assert np.array_equal(eta[-1], V[0] - V[3])
    assert np.array_equal(ux[-1], V[1] / (V[0] + eps))
    assert np.array_equal(uy[-1], V[2] / (V[0] + eps))
    assert np.array_equal(hmax, hm) and np.array_equal(eta_max, em) and np.array_equal(bmin, -bm)
    # the series moved the water at the west boundary, and the mask was used
    assert np.abs(V[0][:, :4] - w.V[0][:, :4]).max() > 1e-3
    V_nomask, _, _ = api_run(None)
    assert not np.array_equal(V_nomask[3], V[3])


def test_tsuner_return_code_3_for_invalid_input(tmp_path, switches):
    w = shelf(10.0, -1.0)
    switches(w.sw)
    bad = w.mask.copy()
    bad[3, 4] = 2  # the mask is 0/1 (Problem_loader.cxx writes only those)
    rc, _ = call_tsuner(w, str(tmp_path / "bad_mask"), mask=bad)
    assert rc == 3
    assert b"mask" in T.lib().tsu_last_error()
    rc, _ = call_tsuner(w, str(tmp_path / "no_series"), with_series=False)  # Read_files = 1 needs the series
    assert rc == 3
    assert not os.path.exists(str(tmp_path / "no_series.nc"))


def test_tsuner_return_code_2_when_the_output_cannot_be_created(tmp_path, switches):
    w = shelf(10.0, -1.0)
    switches(w.sw)
    rc, _ = call_tsuner(w, str(tmp_path / "missing_dir" / "out"))
    assert rc == 2


def test_tsuner_return_code_1_when_gpu_memory_does_not_suffice(tmp_path, switches):
    """Device memory is taken by an ordinary allocation first, so that the
    solver's own allocations fail (cudaErrorMemoryAllocation, no fault)."""
    torch = pytest.importorskip("torch")
    w = shelf(10.0, -1.0)
    switches(w.sw)
    free, _ = torch.cuda.mem_get_info(0)
    hog = torch.empty(max(free - (256 << 20), 0), dtype=torch.uint8, device="cuda:0")
    try:
        big = W.nwave_shelf(2048, 2048, 20.0, slr=0.5, amp=3.0, period=200.0, t_series=100.0)  # ~440 MB on the device
        big.p.total_time, big.p.save_time = 1.0, -1.0
        rc, _ = call_tsuner(big, str(tmp_path / "oom"))
        assert rc == 1
    finally:
        del hog
        torch.cuda.empty_cache()
    rc, _ = call_tsuner(w, str(tmp_path / "after"))  # the device is usable again
    assert rc == 0
