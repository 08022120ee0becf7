"""GPU: the row-slab decomposition through the C ABI (tsu_slab_*) on one
GPU, all slabs held by one process and their ghost rows copied between them
on the device: every owned cell, the running extrema, t and the next dt must
equal, value for value, the undecomposed solver's -- the fused kernels treat
a slab's ghost rows as interior rows and its grid-edge rows as the grid's
boundary.  The multi-GPU transport (NCCL send/recv of the same messages,
MIN all-reduce of the dt) is the path tests/test_slabs_cpu.py runs with gloo."""
import numpy as np
import pytest

import tsuner_b200 as T
from tsuner_b200 import slabs as S
from tsuner_b200 import workloads as W
from tsuner_b200.abi import make_switches

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def cases():
    nw = W.nwave_shelf(512, 384, 10.0, slr=0.5, amp=2.0, period=300.0, t_series=400.0)
    small = W.nwave_shelf(70, 45, 40.0, slr=0.5, amp=2.0, period=300.0, t_series=300.0)
    hump = W.hump(96, 50, 10.0, sigma=80.0)
    return {
        "shelf_series_4_slabs": (nw, nw.sw, 4, 60),
        "shelf_series_3_uneven": (small, small.sw, 3, 80),
        "free_2": (hump, make_switches(order=2, wbc=0, read_files=0), 2, 60),
        "periodic_2": (hump, make_switches(order=2, wbc=2, read_files=0), 2, 60),
        "periodic_series_3": (small, make_switches(order=2, wbc=2, read_files=1), 3, 60),
        # a grid of 2 M cells in 8 slabs (the split of an 8-GPU node), the shelf workload
        "shelf_2048x1024_8_slabs": (big(), big().sw, 8, 40),
    }


_BIG = []


def big():
    if not _BIG:
        _BIG.append(W.nwave_shelf(2048, 1024, 10.0, slr=0.5, amp=3.0, period=300.0, t_series=300.0))
    return _BIG[0]


@pytest.mark.parametrize("name", sorted(cases()))
def test_slabs_equal_the_whole_grid(name):
    w, sw, nslabs, steps = cases()[name]
    s = T.Solver(w.p, sw)
    s.set_state(w.V)
    s.set_mask(w.mask)
    if sw.read_files:
        s.set_boundary_series(w.CC, w.tCC)
    s.reset()
    s.step(steps)
    V_ref = s.state()
    ext_ref = s.extrema()
    t_ref = s.time()
    s.close()

    g = S.SlabGroup(w.p, sw, nslabs=nslabs)
    try:
        g.load(w.V, w.mask, w.CC, w.tCC)
        g.reset()
        g.step(steps)
        g.sync()
        V = np.full_like(V_ref, np.nan)
        for j0, Vs in g.local_state().values():
            V[:, j0:j0 + Vs.shape[1]] = Vs
        for j0, hmax, bmin, eta in g.local_extrema().values():
            rows = slice(j0, j0 + hmax.shape[0])
            assert np.array_equal(hmax, ext_ref[0][rows]) and np.array_equal(bmin, ext_ref[1][rows])
            assert np.array_equal(eta, ext_ref[2][rows])
        assert g.time() == t_ref
    finally:
        g.close()
    assert np.array_equal(V, V_ref), float(np.nanmax(np.abs(V - V_ref)))


def test_slab_refuses_whole_steps_and_bad_rows():
    import ctypes as C
    w = W.hump(64, 40, 10.0)
    p, sw = w.p, w.sw
    h = C.c_void_p()
    L = T.lib()
    assert L.tsu_slab_create(C.byref(h), C.byref(p), C.byref(sw), 0, 1, 0) == T.abi.TSU_ERR_INVALID  # 1 row
    assert L.tsu_slab_create(C.byref(h), C.byref(p), C.byref(sw), 0, 40, 0) == T.abi.TSU_ERR_INVALID  # whole grid
    sw32 = make_switches(order=2, wbc=1, read_files=0, precision=1)
    assert L.tsu_slab_create(C.byref(h), C.byref(p), C.byref(sw32), 0, 20, 0) == T.abi.TSU_ERR_INVALID
    assert L.tsu_slab_create(C.byref(h), C.byref(p), C.byref(sw), 0, 20, 0) == 0
    try:
        assert L.tsu_step(h, 1) == T.abi.TSU_ERR_INVALID
        assert b"slab" in L.tsu_last_error()
    finally:
        L.tsu_destroy(h)
