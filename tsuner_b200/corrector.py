"""Learned corrector: coarse FP32 solves lifted to fine maximum-depth and
bed-change maps by a 6-layer, 32-channel convolutional network trained on
solver-generated fine/coarse pairs.  No counterpart in the reference.

Everything that computes runs in libtsuner_b200.so: the solves (FP32
ensembles for the training pairs and the coarse inputs, the FP64 plain form
for the held-out truth) and the network (tensor-core convolutions, loss and
Adam kernels, tsu_corr_* in include/tsuner_b200.h).  This module only
generates the seeded site and sources and moves arrays through the C ABI.

Site: one fine grid (shelf-to-beach bathymetry with a fractal field and
harbour blocks, +slr sea level); the coarse grid is its `factor` x `factor`
block average (mask: block minimum).  Source k: west-boundary N-wave of
amplitude A_k in [1, 5] m and period T_k in [200, 600] s (seeded).  Sample k
= coarse (maximum depth, bed change, bathymetry) -> fine (maximum depth,
bed change) after `t_end` seconds.  Maximum depth is 0 where a cell was
never wet; bed change is b(t_end) - b(0) = H(0) - H(t_end).
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import Ensemble, Solver, TsunerError, lib
from . import workloads as W
from .abi import make_params, make_switches

LAYERS, CH, KROWS = 6, 32, 288


def _ck(code, what):
    if code != 0:
        detail = lib().tsu_corr_last_error()
        raise TsunerError(code, what + (" [%s]" % detail.decode() if detail else ""))


def _fp(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Corrector:
    """tsu_corr_* handle: fine grid ny x nx, coarse grid (ny/f) x (nx/f)."""

    def __init__(self, ny, nx, factor, max_batch=8, seed=7, device=0):
        self.ny, self.nx, self.f = ny, nx, factor
        self._h = C.c_void_p()
        _ck(lib().tsu_corr_create(C.byref(self._h), ny, nx, factor, max_batch, seed, device), "tsu_corr_create")

    def close(self):
        if self._h:
            lib().tsu_corr_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_site(self, fine_H):
        a = np.ascontiguousarray(fine_H, np.float32).reshape(self.ny, self.nx)
        _ck(lib().tsu_corr_set_site(self._h, _fp(a)), "tsu_corr_set_site")

    def add_samples(self, coarse, fine=None):
        c = np.ascontiguousarray(coarse, np.float32).reshape(-1, 3, self.ny // self.f, self.nx // self.f)
        fi = None if fine is None else np.ascontiguousarray(fine, np.float32).reshape(-1, 2, self.ny, self.nx)
        _ck(lib().tsu_corr_add_samples(self._h, c.shape[0], _fp(c), _fp(fi)), "tsu_corr_add_samples")

    def num_samples(self):
        n = C.c_int()
        _ck(lib().tsu_corr_num_samples(self._h, C.byref(n)), "tsu_corr_num_samples")
        return n.value

    def weights(self):
        Wt = np.empty((LAYERS, CH, 9, CH), np.float32)
        B = np.empty((LAYERS, CH), np.float32)
        _ck(lib().tsu_corr_get_weights(self._h, _fp(Wt), _fp(B)), "tsu_corr_get_weights")
        return Wt, B

    def set_weights(self, Wt, B):
        Wt = np.ascontiguousarray(Wt, np.float32)
        B = np.ascontiguousarray(B, np.float32)
        _ck(lib().tsu_corr_set_weights(self._h, _fp(Wt), _fp(B)), "tsu_corr_set_weights")

    def train(self, ntrain, iters, batch=8, lr=1e-3, seed=1):
        loss = np.empty(max(iters, 1), np.float32)
        _ck(lib().tsu_corr_train(self._h, ntrain, iters, batch, lr, seed, _fp(loss)), "tsu_corr_train")
        return loss[:iters]

    def set_options(self, large_residual_weight=0.0, clip_depth=False, envelope=0.0):
        _ck(lib().tsu_corr_set_options(self._h, float(large_residual_weight), int(bool(clip_depth)), float(envelope)),
            "tsu_corr_set_options")

    def predict(self, first, n):
        shp = (n, self.ny, self.nx)
        oh, ob, bh, bb = (np.empty(shp, np.float32) for _ in range(4))
        _ck(lib().tsu_corr_predict(self._h, first, n, _fp(oh), _fp(ob), _fp(bh), _fp(bb)), "tsu_corr_predict")
        return oh, ob, bh, bb

    def bench_conv(self, nimg, iters):
        ms, tf = C.c_double(), C.c_double()
        _ck(lib().tsu_corr_bench_conv(self._h, nimg, iters, C.byref(ms), C.byref(tf)), "tsu_corr_bench_conv")
        return ms.value, tf.value

    def last_train(self):
        ms, n = C.c_double(), C.c_long()
        _ck(lib().tsu_corr_last_train_ms(self._h, C.byref(ms), C.byref(n)), "tsu_corr_last_train_ms")
        return ms.value, n.value


# ------------------------------------------------------------------ data
@dataclass
class Site:
    n: int           # fine cells per side
    factor: int
    dx: float        # fine cell size (m)
    slr: float
    H: np.ndarray    # fine bathymetry (depth below datum)
    mask: np.ndarray
    Hc: np.ndarray   # coarse bathymetry (block mean)
    maskc: np.ndarray


def block_mean(a, f):
    n0, n1 = a.shape
    return a.reshape(n0 // f, f, n1 // f, f).mean(axis=(1, 3))


def make_site(n=512, factor=4, dx=10.0, slr=0.5, seed=5):
    rng = np.random.default_rng(seed)
    H = W.shelf_bathymetry(n, n, dx, rng, slr)
    mask = W.harbour_mask(n, n, rng)
    Hc = block_mean(H, factor)
    maskc = mask.reshape(n // factor, factor, n // factor, factor).min(axis=(1, 3)).astype(np.int32)
    return Site(n, factor, dx, slr, H, mask, Hc, maskc)


def make_sources(count, seed):
    rng = np.random.default_rng(seed)
    return list(zip(rng.uniform(1.0, 5.0, count), rng.uniform(200.0, 600.0, count)))


def _workload(H, mask, dx, slr, amp, period, t_end, precision):
    n1, n0 = H.shape
    V = np.zeros((5, n1, n0))
    V[0] = np.maximum(slr + H, 0.0)
    V[3] = H
    CC, tCC = W.boundary_series(H, slr, t_end + 20.0, amp=amp, period=period)
    p = make_params(n0, n1, dx, dx)
    sw = make_switches(order=2, wbc=1, read_files=1, precision=precision, eta0=slr)
    return W.Workload("src", p, sw, V, mask, CC, tCC, slr=slr)


def _maps(s, H0):
    hmax, _, _ = s.extrema()
    hmax = np.where(hmax > 0.0, hmax, 0.0)
    H1 = s.state()[3]
    return hmax, H0 - H1


def solve_fp32(H, mask, dx, slr, sources, t_end, chunk=64):
    """Maximum depth and bed change of every source, FP32 ensembles of
    `chunk` members; returns [n][2][ny][nx] float32."""
    out = []
    for k0 in range(0, len(sources), chunk):
        ws = [_workload(H, mask, dx, slr, a, T, t_end, 1) for a, T in sources[k0:k0 + chunk]]
        e = Ensemble([w.p for w in ws], [w.sw for w in ws])
        try:
            e.load(ws)
            e.reset()
            e.run_until(t_end)
            e.sync()
            for s in e.members:
                hm, db = _maps(s, H)
                out.append(np.stack([hm, db]).astype(np.float32))
        finally:
            e.close()
    return np.stack(out)


def solve_fp64(H, mask, dx, slr, sources, t_end):
    """The same maps from the FP64 plain form, one source at a time."""
    out = []
    for a, T in sources:
        w = _workload(H, mask, dx, slr, a, T, t_end, 0)
        s = Solver(w.p, w.sw)
        try:
            s.set_state(w.V)
            s.set_mask(w.mask)
            s.set_boundary_series(w.CC, w.tCC)
            s.reset()
            s.run_until(t_end)
            hm, db = _maps(s, H)
            out.append(np.stack([hm, db]).astype(np.float32))
        finally:
            s.close()
    return np.stack(out)


def coarse_inputs(site, sources, t_end, chunk=128):
    maps = solve_fp32(site.Hc, site.maskc, site.dx * site.factor, site.slr, sources, t_end, chunk)
    Hc = np.broadcast_to(site.Hc.astype(np.float32), (len(sources), 1) + site.Hc.shape)
    return np.concatenate([maps, Hc], axis=1)


def errors(pred, truth, region=None):
    """RMSE and L-inf of maximum depth over `region` (default: cells wet in
    the truth or with a non-zero predicted maximum depth -- a negative one is
    an error too), and RMSE of bed change over all cells.  Pass the same
    region when comparing two predictions so that both RMSEs share one
    denominator."""
    ph, pb = pred
    th, tb = truth[:, 0], truth[:, 1]
    wet = ((th > 0) | (ph != 0)) if region is None else region
    dh = np.where(wet, ph - th, 0.0)
    rm = float(np.sqrt((dh ** 2).sum() / max(wet.sum(), 1)))
    linf = float(np.abs(dh).max())
    rb = float(np.sqrt(((pb - tb) ** 2).mean()))
    return dict(hmax_rmse_m=rm, hmax_linf_m=linf, db_rmse_m=rb)
