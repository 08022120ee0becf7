"""Python bindings of the CPU oracle and of the reference checker builds.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py -- never by the product package.

  liboracle.so            plain-C restatement of the reference step (oracle.c)
  _ref/<v>/libtsuner_ref.so  the reference's own CUDA kernels, unmodified, built
                          per switch variant by build_ref.py and driven by
                          ref_build/ref_harness.cu (needs a GPU)
"""
import ctypes as C
import os

import numpy as np

from tsuner_b200.abi import SimParams, TsuConsts, TsuSwitches

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = {}

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build():
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_consts.argtypes = [C.POINTER(SimParams), C.POINTER(TsuConsts)]
        L.orc_consts.restype = None
        L.orc_initial_dt.argtypes = [C.POINTER(SimParams), C.POINTER(TsuSwitches), _dp, C.c_int]
        L.orc_initial_dt.restype = C.c_double
        L.orc_run.argtypes = [C.POINTER(SimParams), C.POINTER(TsuSwitches), C.c_void_p, _dp, _ip,
                              C.c_void_p, C.c_void_p, C.c_ulong, C.c_void_p, C.c_void_p, C.c_void_p,
                              C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_long, C.c_double, C.c_int,
                              C.c_void_p]
        L.orc_run.restype = C.c_long
        L.orc_init_extrema.argtypes = [C.c_long, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_max_threads.restype = C.c_int
        L.orc_slab_stage.argtypes = [C.POINTER(SimParams), C.POINTER(TsuSwitches), C.c_void_p] + [C.c_int] * 5 + \
            [C.c_void_p] * 6 + [C.c_ulong, C.c_double, C.c_double, C.c_int]
        L.orc_slab_stage.restype = C.c_int
        L.orc_slab_dt.argtypes = [C.POINTER(SimParams), C.POINTER(TsuSwitches)] + [C.c_int] * 4 + [C.c_void_p]
        L.orc_slab_dt.restype = C.c_double
        L.orc_slab_extrema.argtypes = [C.POINTER(SimParams)] + [C.c_int] * 4 + [C.c_void_p] * 4
        L.orc_slab_extrema.restype = None
        _LIB = L
    return _LIB


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def consts(p):
    k = TsuConsts()
    lib().orc_consts(C.byref(p), C.byref(k))
    return k


def max_threads():
    return lib().orc_max_threads()


def initial_dt(p, sw, V, nthreads=0):
    return lib().orc_initial_dt(C.byref(p), C.byref(sw), np.ascontiguousarray(V, np.float64), nthreads)


class OracleRun:
    """Host state for the oracle: V (5, npy, npx) SoA, extrema, t, dt."""

    def __init__(self, p, sw, V, mask=None, CC=None, tCC=None, kconsts=None, nthreads=0):
        self.p, self.sw = p, sw
        n = p.npx * p.npy
        self.V = np.ascontiguousarray(V, np.float64).reshape(5, p.npy, p.npx).copy()
        self.mask = (np.ones(n, np.int32) if mask is None
                     else np.ascontiguousarray(mask, np.int32).reshape(-1).copy())
        self.CC = None if CC is None else np.ascontiguousarray(CC, np.float64)
        self.tCC = None if tCC is None else np.ascontiguousarray(tCC, np.float64)
        self.timeCC = 0 if tCC is None else len(self.tCC)
        self.k = kconsts
        self.nthreads = nthreads
        self.hmax = np.empty(n)
        self.bmin = np.empty(n)
        self.eta_max = np.empty(n)
        lib().orc_init_extrema(n, _ptr(self.hmax), _ptr(self.bmin), _ptr(self.eta_max))
        self.t = C.c_double(0.0)
        self.dt = C.c_double(-1.0)
        self.steps = 0
        # MUSCL-Hancock's unfiltered working state, carried across run() calls
        self.Vk = self.V.copy()

    def run(self, nsteps=-1, t_end=0.0):
        k = None if self.k is None else C.byref(self.k)
        n = lib().orc_run(C.byref(self.p), C.byref(self.sw), k, self.V.reshape(-1), self.mask,
                          _ptr(self.CC), _ptr(self.tCC), self.timeCC, _ptr(self.hmax),
                          _ptr(self.bmin), _ptr(self.eta_max), C.byref(self.t), C.byref(self.dt),
                          nsteps, t_end, self.nthreads, _ptr(self.Vk))
        if n < 0:
            raise RuntimeError("oracle run failed (%d)" % n)
        self.steps += n
        return n


class OracleSlab:
    """A row slab stepped by the oracle on the host: the compute backend that
    the CPU tests of tsuner_b200.slabs.SlabGroup put in place of the device
    (same calls as DeviceSlab; messages are CPU torch tensors, so a gloo
    group carries them).  It keeps the reference's three state arrays V, V0,
    Vk for the stored rows; both state buffers of the device (the state a
    step starts from, the intermediate RK state) are V here, as in the
    reference, whose V holds whichever state the next stage reads."""

    def __init__(self, p, sw, j0, j1, device=None, kconsts=None):
        import torch
        self.torch = torch
        self.p, self.sw, self.j0, self.j1, self.k = p, sw, j0, j1, kconsts
        periodic = sw.wbc == 2
        self.gs = 2 if (j0 > 0 or periodic) else 0
        self.gn = 2 if (j1 < p.npy or periodic) else 0
        self.n = j1 - j0
        nst = self.gs + self.n + self.gn
        self.V = np.zeros((5, nst, p.npx))
        self.V0 = np.zeros_like(self.V)
        self.Vk = np.zeros_like(self.V)
        self.mask = np.ones((nst, p.npx), np.int32)
        self.ext = [np.full((nst, p.npx), -1e30) for _ in range(3)]
        self.CC = self.tCC = None
        self.timeCC = 0
        self.t, self.dt, self.dt_local, self.steps = 0.0, -1.0, -1.0, 0
        self._recv = {}
        for which in (0, 1, 2):
            planes = 1 if which == 2 else 5
            for side in (0, 1):
                self._recv[which, side] = torch.empty(planes * 2 * p.npx,
                                                      dtype=torch.uint8 if which == 2 else torch.float64)

    def _rows(self, side, ghost):
        if ghost:
            return slice(0, 2) if side == 0 else slice(self.gs + self.n, self.gs + self.n + 2)
        return slice(self.gs, self.gs + 2) if side == 0 else slice(self.gs + self.n - 2, self.gs + self.n)

    def _slab_args(self):
        return (self.j0, self.j1, self.gs, self.gn)

    def set_state(self, V):
        self.V[:, self.gs:self.gs + self.n] = V

    def set_mask(self, mask):
        self.mask[self.gs:self.gs + self.n] = 1 if mask is None else mask

    def set_boundary_series(self, CC, tCC):
        self.CC = np.ascontiguousarray(CC, np.float64)
        self.tCC = np.ascontiguousarray(tCC, np.float64)
        self.timeCC = len(self.tCC)

    def reset(self):
        self.t, self.steps = 0.0, 0
        for e in self.ext:
            e[:] = -1e30
        self.V0[:] = self.V
        self.Vk[:] = self.V
        self.dt_local = lib().orc_slab_dt(C.byref(self.p), C.byref(self.sw), *self._slab_args(), _ptr(self.V))

    def stage(self, k):
        kk = None if self.k is None else C.byref(self.k)
        rc = lib().orc_slab_stage(C.byref(self.p), C.byref(self.sw), kk, *self._slab_args(), k, _ptr(self.V),
                                  _ptr(self.V0), _ptr(self.Vk), _ptr(self.mask), _ptr(self.CC), _ptr(self.tCC),
                                  self.timeCC, self.t, self.dt, 0)
        if rc:
            raise RuntimeError("oracle slab stage failed (%d)" % rc)
        if k == self.sw.order - 1:  # the end of the step (GPU/main_TSUNER.cu:185-192)
            self.t += self.dt
            self.steps += 1
            lib().orc_slab_extrema(C.byref(self.p), *self._slab_args(), _ptr(self.V), *[_ptr(e) for e in self.ext])
            self.dt_local = lib().orc_slab_dt(C.byref(self.p), C.byref(self.sw), *self._slab_args(), _ptr(self.V))

    def pack(self, which, side):
        rows = self._rows(side, ghost=False)
        src = self.mask[rows].astype(np.uint8) if which == 2 else self.V[:, rows]
        return self.torch.from_numpy(np.ascontiguousarray(src).reshape(-1).copy())

    def recv_buffer(self, which, side):
        return self._recv[which, side]

    def unpack(self, which, side):
        rows = self._rows(side, ghost=True)
        buf = self._recv[which, side].numpy()
        if which == 2:
            self.mask[rows] = buf.reshape(2, self.p.npx)
        else:
            self.V[:, rows] = buf.reshape(5, 2, self.p.npx)

    def dt_buffer(self):
        return self.torch.tensor([self.dt_local], dtype=self.torch.float64)

    def set_dt(self, d):
        self.dt = float(d[0])

    def sync(self):
        pass

    def state(self):
        return self.V[:, self.gs:self.gs + self.n].copy()

    def extrema(self):
        return tuple(e[self.gs:self.gs + self.n].copy() for e in self.ext)

    def time(self):
        return self.t, self.dt, self.steps


# ---------------------------------------------------------------- reference
def ref_path(variant="default"):
    return os.path.join(HERE, "_ref", variant, "libtsuner_ref.so")


def ref_available(variant="default"):
    return os.path.exists(ref_path(variant))


def ref_lib(variant="default"):
    if variant not in _REF:
        L = C.CDLL(ref_path(variant))
        L.ref_run.argtypes = [SimParams, _dp, _ip, C.c_void_p, C.c_void_p, C.c_ulong, C.c_long,
                              C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double),
                              C.POINTER(C.c_double), C.POINTER(C.c_long), C.POINTER(C.c_double), C.c_int]
        L.ref_run.restype = C.c_int
        L.ref_switches.argtypes = [_ip]
        L.ref_initial_dt.argtypes = [SimParams, _dp, C.POINTER(C.c_double), C.c_int]
        _REF[variant] = L
    return _REF[variant]


def ref_gpu_count(variant="default"):
    """CUDA devices visible to the reference build (0 without a GPU or driver);
    asks the reference library's own CUDA runtime, so the product library is
    not loaded."""
    if not ref_available(variant):
        return 0
    L = ref_lib(variant)
    f = getattr(L, "ref_device_count", None) or getattr(L, "cudaGetDeviceCount", None)
    if f is None:
        return 0
    n = C.c_int(0)
    f.argtypes = [C.POINTER(C.c_int)]
    f.restype = C.c_int
    return n.value if f(C.byref(n)) == 0 else 0


def ref_switches(variant="default"):
    out = np.zeros(6, np.int32)
    ref_lib(variant).ref_switches(out)
    return dict(zip(("order", "rk", "wbc", "bedload", "suspension", "read_files"), out.tolist()))


def ref_run(variant, p, V, mask=None, CC=None, tCC=None, nsteps=1, device=0, work=None, ext=None):
    """Runs the reference build for nsteps; returns dict with V, extrema, t, dt, ms.
    work: optional float64 buffer of 5*npx*npy elements that holds the state
    on entry and receives it on return (used in place, e.g. pinned memory);
    ext: optional three buffers of npx*npy doubles for the extrema."""
    n = p.npx * p.npy
    if work is None:
        Vh = np.ascontiguousarray(V, np.float64).reshape(-1).copy()
    else:
        Vh = work.reshape(-1)
        assert Vh.dtype == np.float64 and Vh.size == 5 * n and Vh.flags.c_contiguous
    m = np.ones(n, np.int32) if mask is None else np.ascontiguousarray(mask, np.int32).reshape(-1)
    hmax, bmin, eta = (np.empty(n), np.empty(n), np.empty(n)) if ext is None else (e.reshape(-1) for e in ext)
    t, dt, ms = C.c_double(), C.c_double(), C.c_double()
    steps = C.c_long()
    CCa = None if CC is None else np.ascontiguousarray(CC, np.float64)
    tCa = None if tCC is None else np.ascontiguousarray(tCC, np.float64)
    rc = ref_lib(variant).ref_run(p, Vh, m, _ptr(CCa), _ptr(tCa), 0 if tCa is None else len(tCa),
                                  nsteps, _ptr(hmax), _ptr(bmin), _ptr(eta), C.byref(t),
                                  C.byref(dt), C.byref(steps), C.byref(ms), device)
    if rc != 0:
        raise RuntimeError("reference harness failed (%d)" % rc)
    return dict(V=Vh.reshape(5, p.npy, p.npx), hmax=hmax.reshape(p.npy, p.npx),
                bmin=bmin.reshape(p.npy, p.npx), eta_max=eta.reshape(p.npy, p.npx),
                t=t.value, dt=dt.value, ms=ms.value, steps=steps.value)
