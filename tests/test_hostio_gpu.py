"""GPU: bulk host <-> device copies of the C ABI (tsu_copy_* and the
tsu_set_* / tsu_get_* calls built on them).  Bytes must arrive unchanged on
every path: small copies handed to the driver, pageable buffers staged
through the pinned chunks (several chunks per plane, more chunks than
buffers, rows that do not divide a chunk), pinned host buffers copied
directly, pitched host and device rows, flat ranges with odd tails, and
destinations the process has never touched.  Device row padding stays as it
was."""
import ctypes as C

import numpy as np
import pytest

import tsuner_b200 as T
from tsuner_b200.abi import TSU_ERR_INVALID, make_params, make_switches

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def ptrs(items):
    return (C.c_void_p * len(items))(*[C.c_void_p(p) for p in items])


def host_addr(a):
    return a.ctypes.data


def rand_bytes(n, seed):
    return np.random.default_rng(seed).integers(0, 256, n, dtype=np.uint8)


@pytest.mark.parametrize("nplanes,width,rows,hpitch,dpitch", [
    (3, 8000, 2100, 8000, 8192),   # 16.8 MB planes: 2 chunks each, 6 chunks over 4 buffers
    (2, 8000, 2100, 8064, 8192),   # pitched host rows
    (1, 300, 700, 300, 512),       # 210 KB: driver path
    (5, 4096 * 8, 1025, 4096 * 8, 4096 * 8 + 512),  # 512 rows per chunk, 3 chunks per plane
])
def test_planes_round_trip(nplanes, width, rows, hpitch, dpitch):
    d = dev()
    L = T.lib()
    src = [rand_bytes(rows * hpitch, 10 + k) for k in range(nplanes)]
    D = torch.full((nplanes, rows * dpitch), 0xAB, dtype=torch.uint8, device=d)
    torch.cuda.synchronize()
    dptr = [D[k].data_ptr() for k in range(nplanes)]
    rc = L.tsu_copy_planes_to_device(0, nplanes, ptrs(dptr), dpitch, ptrs([host_addr(a) for a in src]), hpitch,
                                     width, rows)
    assert rc == 0, L.tsu_last_error()
    got = D.cpu().numpy().reshape(nplanes, rows, dpitch)
    for k in range(nplanes):
        want = src[k].reshape(rows, hpitch)[:, :width]
        assert np.array_equal(got[k, :, :width], want)
        assert (got[k, :, width:] == 0xAB).all()  # device row padding untouched
    back = [np.empty(rows * hpitch, np.uint8) for _ in range(nplanes)]  # never touched before the copy
    rc = L.tsu_copy_planes_to_host(0, nplanes, ptrs([host_addr(a) for a in back]), hpitch, ptrs(dptr), dpitch,
                                   width, rows)
    assert rc == 0, L.tsu_last_error()
    for k in range(nplanes):
        assert np.array_equal(back[k].reshape(rows, hpitch)[:, :width], src[k].reshape(rows, hpitch)[:, :width])


def test_pinned_host_planes():
    d = dev()
    L = T.lib()
    nplanes, width, rows = 2, 8000, 2100
    pin = torch.empty((nplanes, rows * width), dtype=torch.uint8, pin_memory=True)
    src = pin.numpy()
    src[...] = rand_bytes(src.size, 3).reshape(src.shape)
    D = torch.zeros((nplanes, rows * width), dtype=torch.uint8, device=d)
    torch.cuda.synchronize()
    dptr = [D[k].data_ptr() for k in range(nplanes)]
    hptr = [src[k].ctypes.data for k in range(nplanes)]
    assert L.tsu_copy_planes_to_device(0, nplanes, ptrs(dptr), width, ptrs(hptr), width, width, rows) == 0
    assert np.array_equal(D.cpu().numpy(), src)
    out = torch.zeros((nplanes, rows * width), dtype=torch.uint8, pin_memory=True).numpy()
    optr = [out[k].ctypes.data for k in range(nplanes)]
    assert L.tsu_copy_planes_to_host(0, nplanes, ptrs(optr), width, ptrs(dptr), width, width, rows) == 0
    assert np.array_equal(out, src)


@pytest.mark.parametrize("nbytes", [0, 1, 65535, 65536, (1 << 20) + 7, (16 << 20) + 3, (50 << 20) + 12345])
def test_bytes_round_trip(nbytes):
    d = dev()
    L = T.lib()
    src = rand_bytes(nbytes, nbytes % 1000)
    D = torch.full((nbytes + 64,), 0x5A, dtype=torch.uint8, device=d)
    torch.cuda.synchronize()
    assert L.tsu_copy_bytes_to_device(0, C.c_void_p(D.data_ptr()), C.c_void_p(host_addr(src)), nbytes) == 0
    got = D.cpu().numpy()
    assert np.array_equal(got[:nbytes], src) and (got[nbytes:] == 0x5A).all()
    back = np.empty(nbytes, np.uint8)
    assert L.tsu_copy_bytes_to_host(0, C.c_void_p(host_addr(back)), C.c_void_p(D.data_ptr()), nbytes) == 0
    assert np.array_equal(back, src)


def test_copy_arguments_rejected():
    d = dev()
    L = T.lib()
    D = torch.zeros(4096, dtype=torch.uint8, device=d)
    h = np.zeros(4096, np.uint8)
    one_d, one_h = ptrs([D.data_ptr()]), ptrs([host_addr(h)])
    assert L.tsu_copy_planes_to_device(0, 1, one_d, 64, one_h, 128, 128, 4) == TSU_ERR_INVALID  # width > pitch
    assert L.tsu_copy_planes_to_host(0, 1, ptrs([0]), 64, one_d, 64, 64, 4) == TSU_ERR_INVALID  # NULL plane
    assert L.tsu_copy_bytes_to_device(0, None, C.c_void_p(host_addr(h)), 16) == TSU_ERR_INVALID


def _solver(npx, npy, precision):
    p = make_params(npx, npy, 5.0, 5.0)
    sw = make_switches(order=2, wbc=1, read_files=0, precision=precision, eta0=0.5)
    return T.Solver(p, sw)


def test_state_round_trip_fp64_padded_rows():
    """FP64 set_state / get_state at a width whose device rows are padded:
    the state comes back bit for bit (no step in between)."""
    dev()
    npx, npy = 1000, 1100  # 8.8 MB per plane, device pitch > npx
    rng = np.random.default_rng(1)
    V = np.abs(rng.normal(1.0, 0.5, (5, npy, npx)))
    s = _solver(npx, npy, 0)
    try:
        s.set_state(V)
        assert np.array_equal(s.state(), V)
    finally:
        s.close()


def test_mask_bad_value_reported_at_its_index():
    dev()
    npx, npy = 640, 480
    s = _solver(npx, npy, 1)
    try:
        m = np.ones((npy, npx), np.int32)
        m[npy - 1, npx - 1] = 2
        with pytest.raises(T.TsunerError) as e:
            s.set_mask(m)
        assert "at %d" % (npx * npy - 1) in str(e.value)
        m[npy - 1, npx - 1] = 1
        m[3, 5] = -1
        with pytest.raises(T.TsunerError) as e:
            s.set_mask(m)
        assert "at %d" % (3 * npx + 5) in str(e.value)
        m[3, 5] = 0
        s.set_mask(m)  # a valid mask is accepted afterwards
    finally:
        s.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_boundary_series_replaced_in_place(precision):
    """The boundary series buffers are kept across tsu_set_boundary_series
    calls and only grown.  A series replaced by a shorter one, and a short
    one replaced by a longer one (with steps of the old series still queued
    on the solver's stream), must step exactly like a fresh solver given only
    the final series."""
    dev()
    from tsuner_b200 import workloads as W
    w = W.nwave_shelf(npx=256, npy=192, steps=40)
    H = w.V[3]
    long_s = W.boundary_series(H, w.slr, 4000.0, amp=3.0, period=600.0)  # ~23 MB: staged upload
    short_s = W.boundary_series(H, w.slr, 500.0, amp=2.0, period=300.0)
    sw = make_switches(order=2, wbc=1, read_files=1, precision=precision, eta0=w.slr)

    def run(series_list):
        s = T.Solver(w.p, sw)
        try:
            for k, (CC, tCC) in enumerate(series_list):
                s.set_state(w.V)
                s.set_mask(w.mask)
                s.set_boundary_series(CC, tCC)
                s.reset()
                s.step(5 if k + 1 < len(series_list) else 40)
            return s.state(), s.time()
        finally:
            s.close()

    for first, final in ((long_s, short_s), (short_s, long_s)):
        V1, t1 = run([first, final])
        V0, t0 = run([final])
        assert np.array_equal(V1, V0)
        assert t1 == t0
    # the two series really give different runs
    Va, _ = run([long_s])
    Vb, _ = run([short_s])
    assert not np.array_equal(Va, Vb)
