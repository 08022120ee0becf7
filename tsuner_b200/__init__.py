"""tsuner_b200 -- B200-native TSUNER hot path behind a C ABI.

The product is the shared library libtsuner_b200.so (hand-written sm_100a
CUDA + C++ host code) declared by include/tsuner_b200.h.  This module is a
thin ctypes binding over that ABI for tests and benchmarks; it has no
compute of its own and no CPU fallback: if the library is missing or cannot
be loaded the import of `lib()` raises.
"""
import ctypes as C
import os

import numpy as np

from .abi import (SimParams, TsuConsts, TsuSwitches, TSU_OK, make_params,  # noqa: F401
                  make_switches, derive_params)

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libtsuner_b200.so")
_LIB = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")

# every symbol include/tsuner_b200.h declares
EXPORTS = [
    "TSUNER", "checkCUDAsupport", "initializeGPU",
    "tsu_switches_default", "tsu_set_default_switches", "tsu_get_default_switches",
    "tsu_derive_params", "tsu_parse_data_dat",
    "tsu_create", "tsu_destroy", "tsu_set_state", "tsu_set_mask", "tsu_set_boundary_series",
    "tsu_reset", "tsu_resume", "tsu_step", "tsu_run_until", "tsu_sync", "tsu_get_state", "tsu_get_extrema",
    "tsu_get_time", "tsu_get_sums", "tsu_get_consts", "tsu_last_step_ms", "tsu_last_step_launches",
    "tsu_state_device", "tsu_cfl_dt_noalloc", "tsu_copy_planes_to_device", "tsu_copy_planes_to_host",
    "tsu_copy_bytes_to_device", "tsu_copy_bytes_to_host", "tsu_host_threads", "tsu_strerror", "tsu_last_error",
    "tsu_version", "tsu_struct_sizes",
    "tsu_ens_create", "tsu_ens_destroy", "tsu_ens_member", "tsu_ens_reset", "tsu_ens_step", "tsu_ens_sync",
    "tsu_ens_autotune", "tsu_ens_set_config", "tsu_ens_get_config", "tsu_ens_last_step_ms",
    "tsu_ens_last_step_launches", "tsu_ens_run_until",
    "tsu_corr_create", "tsu_corr_destroy", "tsu_corr_set_site", "tsu_corr_add_samples", "tsu_corr_num_samples",
    "tsu_corr_get_weights", "tsu_corr_set_weights", "tsu_corr_train", "tsu_corr_set_options", "tsu_corr_predict",
    "tsu_corr_bench_conv",
    "tsu_corr_last_train_ms", "tsu_corr_conv3x3", "tsu_corr_conv3x3_wgrad", "tsu_corr_status",
    "tsu_corr_last_error", "tsu_set_wait_limit_ns",
    "tsu_slab_create", "tsu_slab_info", "tsu_slab_halo_bytes", "tsu_slab_pack", "tsu_slab_unpack", "tsu_slab_stage",
    "tsu_get_dt_device", "tsu_set_dt_device", "tsu_set_stream",
    "tsu_nctr_interp_grid", "tsu_nctr_fix_eta", "tsu_nctr_boundary_series", "tsu_nctr_sphere_metrics",
    "tsu_nctr_to_cartesian", "tsu_nctr_to_cartesian_series", "tsu_nctr_assign_state", "tsu_nctr_prepare",
    "tsu_nctr_tides",
]

_ENS_SIG = {
    "tsu_ens_create": ([C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int], C.c_int),
    "tsu_ens_destroy": ([C.c_void_p], C.c_int),
    "tsu_ens_member": ([C.c_void_p, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "tsu_ens_reset": ([C.c_void_p], C.c_int),
    "tsu_ens_step": ([C.c_void_p, C.c_long], C.c_int),
    "tsu_ens_sync": ([C.c_void_p], C.c_int),
    "tsu_ens_autotune": ([C.c_void_p, C.c_int, C.c_char_p, C.c_size_t], C.c_int),
    "tsu_ens_set_config": ([C.c_void_p, C.c_int, C.c_int, C.c_int], C.c_int),
    "tsu_ens_get_config": ([C.c_void_p] + [C.POINTER(C.c_int)] * 5 + [C.POINTER(C.c_long)], C.c_int),
    "tsu_ens_last_step_ms": ([C.c_void_p, C.POINTER(C.c_double)], C.c_int),
    "tsu_ens_last_step_launches": ([C.c_void_p, C.POINTER(C.c_long)], C.c_int),
    "tsu_ens_run_until": ([C.c_void_p, C.c_double, C.c_long, C.POINTER(C.c_long)], C.c_int),
    "tsu_corr_create": ([C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.c_int],
                        C.c_int),
    "tsu_corr_destroy": ([C.c_void_p], C.c_int),
    "tsu_corr_set_site": ([C.c_void_p, C.c_void_p], C.c_int),
    "tsu_corr_add_samples": ([C.c_void_p, C.c_int, C.c_void_p, C.c_void_p], C.c_int),
    "tsu_corr_num_samples": ([C.c_void_p, C.POINTER(C.c_int)], C.c_int),
    "tsu_corr_get_weights": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "tsu_corr_set_weights": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "tsu_corr_train": ([C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_ulonglong, C.c_void_p], C.c_int),
    "tsu_corr_predict": ([C.c_void_p, C.c_int, C.c_int] + [C.c_void_p] * 4, C.c_int),
    "tsu_corr_set_options": ([C.c_void_p, C.c_float, C.c_int, C.c_float], C.c_int),
    "tsu_corr_bench_conv": ([C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int),
    "tsu_corr_last_train_ms": ([C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_long)], C.c_int),
    "tsu_corr_conv3x3": ([C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                          C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "tsu_corr_conv3x3_wgrad": ([C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                C.c_void_p], C.c_int),
    "tsu_corr_status": ([], C.c_int),
    "tsu_corr_last_error": ([], C.c_char_p),
}


class TsunerError(RuntimeError):
    def __init__(self, code, what):
        msg = "%s failed: %s (%d)" % (what, lib().tsu_strerror(code).decode(), code)
        detail = lib().tsu_last_error()
        if detail:
            msg += " -- " + detail.decode()
        super().__init__(msg)
        self.code = code


def lib():
    """Loads the product library (raises if it is not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libtsuner_b200.so is not built; run `python -m tsuner_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        sig = {
            "tsu_switches_default": ([C.POINTER(TsuSwitches)], C.c_int),
            "tsu_set_default_switches": ([C.POINTER(TsuSwitches)], C.c_int),
            "tsu_get_default_switches": ([C.POINTER(TsuSwitches)], C.c_int),
            "tsu_derive_params": ([C.POINTER(SimParams), C.c_double], C.c_int),
            "tsu_create": ([C.POINTER(vp), C.POINTER(SimParams), C.POINTER(TsuSwitches), C.c_int], C.c_int),
            "tsu_destroy": ([vp], C.c_int),
            "tsu_set_state": ([vp, vp, vp, vp, vp, vp], C.c_int),
            "tsu_set_mask": ([vp, vp], C.c_int),
            "tsu_set_boundary_series": ([vp, vp, vp, C.c_ulong], C.c_int),
            "tsu_reset": ([vp], C.c_int),
            "tsu_resume": ([vp, C.c_double, C.c_long, vp, vp, vp], C.c_int),
            "tsu_step": ([vp, C.c_long], C.c_int),
            "tsu_run_until": ([vp, C.c_double, C.c_long, C.POINTER(C.c_long)], C.c_int),
            "tsu_sync": ([vp], C.c_int),
            "tsu_get_state": ([vp, vp], C.c_int),
            "tsu_get_extrema": ([vp, vp, vp, vp], C.c_int),
            "tsu_get_time": ([vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_long)], C.c_int),
            "tsu_get_consts": ([vp, C.POINTER(TsuConsts)], C.c_int),
            "tsu_get_sums": ([vp, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int),
            "tsu_last_step_ms": ([vp, C.POINTER(C.c_double)], C.c_int),
            "tsu_last_step_launches": ([vp, C.POINTER(C.c_long)], C.c_int),
            "tsu_state_device": ([vp, C.POINTER(vp), C.POINTER(C.c_long), C.POINTER(C.c_long),
                                  C.POINTER(C.c_int)], C.c_int),
            "tsu_cfl_dt_noalloc": ([vp, vp, vp, C.c_long, C.POINTER(SimParams), vp, vp], C.c_int),
            "tsu_copy_planes_to_device": ([C.c_int, C.c_int, C.POINTER(vp), C.c_size_t, C.POINTER(vp), C.c_size_t,
                                           C.c_size_t, C.c_size_t], C.c_int),
            "tsu_copy_planes_to_host": ([C.c_int, C.c_int, C.POINTER(vp), C.c_size_t, C.POINTER(vp), C.c_size_t,
                                         C.c_size_t, C.c_size_t], C.c_int),
            "tsu_copy_bytes_to_device": ([C.c_int, vp, vp, C.c_size_t], C.c_int),
            "tsu_copy_bytes_to_host": ([C.c_int, vp, vp, C.c_size_t], C.c_int),
            "tsu_host_threads": ([], C.c_int),
            "tsu_strerror": ([C.c_int], C.c_char_p),
            "tsu_last_error": ([], C.c_char_p),
            "tsu_version": ([], C.c_char_p),
            "tsu_struct_sizes": ([C.POINTER(C.c_size_t)], C.c_int),
            "tsu_parse_data_dat": ([C.c_char_p, C.POINTER(SimParams), C.c_char_p, C.c_char_p, C.c_char_p,
                                    C.c_char_p, C.POINTER(C.c_double), C.c_char_p, C.c_size_t], C.c_int),
            "tsu_set_wait_limit_ns": ([C.c_ulonglong], C.c_int),
            "tsu_slab_create": ([C.POINTER(vp), C.POINTER(SimParams), C.POINTER(TsuSwitches), C.c_int, C.c_int,
                                 C.c_int], C.c_int),
            "tsu_slab_info": ([vp] + [C.POINTER(C.c_int)] * 4, C.c_int),
            "tsu_slab_halo_bytes": ([vp, C.c_int, C.POINTER(C.c_size_t)], C.c_int),
            "tsu_slab_pack": ([vp, C.c_int, C.c_int, vp], C.c_int),
            "tsu_slab_unpack": ([vp, C.c_int, C.c_int, vp], C.c_int),
            "tsu_slab_stage": ([vp, C.c_int], C.c_int),
            "tsu_get_dt_device": ([vp, vp], C.c_int),
            "tsu_set_dt_device": ([vp, vp], C.c_int),
            "tsu_set_stream": ([vp, vp], C.c_int),
            "tsu_nctr_interp_grid": ([C.c_double] * 6 + [C.c_int] * 2 + [C.c_double] * 2 + [C.c_int] * 2 + [vp, vp],
                                     C.c_int),
            "tsu_nctr_fix_eta": ([vp, vp, C.c_int, C.c_int, C.c_double], C.c_int),
            "tsu_nctr_boundary_series": ([vp, vp, vp, C.c_ulong, C.c_int, C.c_int] + [C.c_double] * 4 +
                                         [C.c_int] * 2 + [C.c_double] * 4 + [vp, C.c_double, vp], C.c_int),
            "tsu_nctr_sphere_metrics": ([C.c_double, C.c_double, C.c_int, C.c_double, C.c_double, C.c_double,
                                         vp, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int),
            "tsu_nctr_to_cartesian": ([C.c_double] * 4 + [vp, C.c_double, C.c_int, C.c_int, vp, vp], C.c_int),
            "tsu_nctr_to_cartesian_series": ([C.c_double] * 4 + [vp, C.c_double, C.c_int, C.c_int, C.c_ulong, vp],
                                             C.c_int),
            "tsu_nctr_assign_state": ([vp, vp, vp, C.c_int, C.c_int, C.c_double, vp, vp, vp, vp], C.c_int),
            "tsu_nctr_prepare": ([C.c_int, C.c_int, vp, vp, vp, C.c_int, C.c_int, vp, vp, vp, C.c_int, C.c_int, vp,
                                  vp, C.c_ulong, vp, vp, vp, vp, C.c_int, C.c_int, C.c_double,
                                  C.POINTER(SimParams), vp, vp, vp, vp, vp, vp], C.c_int),
            "tsu_nctr_tides": ([vp, C.c_int, C.c_int, C.c_ulong, vp, C.c_int, C.c_int] + [C.c_double] * 4 + [vp],
                               C.c_int),
            "checkCUDAsupport": ([C.c_int], C.c_int),
            "initializeGPU": ([], None),
        }
        sig.update(_ENS_SIG)
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _LIB = L
    return _LIB


def _ck(code, what):
    if code != TSU_OK:
        raise TsunerError(code, what)


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Solver:
    """One simulation on one GPU through the tsu_* C ABI."""

    def __init__(self, p, sw, device=0):
        self.p, self.sw = p, sw
        self._h = C.c_void_p()
        _ck(lib().tsu_create(C.byref(self._h), C.byref(p), C.byref(sw), device), "tsu_create")

    @classmethod
    def _borrow(cls, handle, p, sw):
        """View of a solver owned by someone else (an ensemble member)."""
        s = cls.__new__(cls)
        s.p, s.sw, s._h, s._owned = p, sw, handle, False
        return s

    def close(self):
        if self._h and getattr(self, "_owned", True):
            lib().tsu_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_state(self, V):
        V = np.ascontiguousarray(V, np.float64).reshape(5, self.p.npy, self.p.npx)
        _ck(lib().tsu_set_state(self._h, _p(V[0]), _p(V[1]), _p(V[2]), _p(V[3]), _p(V[4])), "tsu_set_state")

    def set_mask(self, mask):
        m = None if mask is None else np.ascontiguousarray(mask, np.int32).reshape(-1)
        _ck(lib().tsu_set_mask(self._h, _p(m)), "tsu_set_mask")

    def set_boundary_series(self, CC, tCC):
        self._CC = np.ascontiguousarray(CC, np.float64)
        self._tCC = np.ascontiguousarray(tCC, np.float64)
        _ck(lib().tsu_set_boundary_series(self._h, _p(self._CC), _p(self._tCC), len(self._tCC)),
            "tsu_set_boundary_series")

    def reset(self):
        _ck(lib().tsu_reset(self._h), "tsu_reset")

    def resume(self, t, steps, extrema=None):
        """Continue a checkpoint after set_state / set_mask / set_boundary_series
        / reset: the saved (t, steps) of time() and optionally the saved
        (hmax, bmin, eta_max) of extrema()."""
        ex = [None] * 3 if extrema is None else [None if e is None else np.ascontiguousarray(e, np.float64)
                                                 for e in extrema]
        _ck(lib().tsu_resume(self._h, float(t), int(steps), *[_p(e) for e in ex]), "tsu_resume")

    def step(self, n):
        _ck(lib().tsu_step(self._h, n), "tsu_step")

    def run_until(self, t_end, max_steps=1 << 40):
        n = C.c_long()
        _ck(lib().tsu_run_until(self._h, t_end, max_steps, C.byref(n)), "tsu_run_until")
        return n.value

    def sync(self):
        _ck(lib().tsu_sync(self._h), "tsu_sync")

    def state(self):
        V = np.empty((5, self.p.npy, self.p.npx))
        _ck(lib().tsu_get_state(self._h, _p(V)), "tsu_get_state")
        return V

    def extrema(self):
        shp = (self.p.npy, self.p.npx)
        a, b, c = np.empty(shp), np.empty(shp), np.empty(shp)
        _ck(lib().tsu_get_extrema(self._h, _p(a), _p(b), _p(c)), "tsu_get_extrema")
        return a, b, c

    def time(self):
        t, dt, n = C.c_double(), C.c_double(), C.c_long()
        _ck(lib().tsu_get_time(self._h, C.byref(t), C.byref(dt), C.byref(n)), "tsu_get_time")
        return t.value, dt.value, n.value

    def sums(self):
        """FP32 form: FP64 (sum of h, sum of H + hc) over the grid."""
        a, b = C.c_double(), C.c_double()
        _ck(lib().tsu_get_sums(self._h, C.byref(a), C.byref(b)), "tsu_get_sums")
        return a.value, b.value

    def consts(self):
        k = TsuConsts()
        _ck(lib().tsu_get_consts(self._h, C.byref(k)), "tsu_get_consts")
        return k

    def last_ms(self):
        ms = C.c_double()
        _ck(lib().tsu_last_step_ms(self._h, C.byref(ms)), "tsu_last_step_ms")
        return ms.value

    def last_launches(self):
        n = C.c_long()
        _ck(lib().tsu_last_step_launches(self._h, C.byref(n)), "tsu_last_step_launches")
        return n.value

    def device_state(self):
        ptr, pitch, plane, eb = C.c_void_p(), C.c_long(), C.c_long(), C.c_int()
        _ck(lib().tsu_state_device(self._h, C.byref(ptr), C.byref(pitch), C.byref(plane), C.byref(eb)),
            "tsu_state_device")
        return ptr.value, pitch.value, plane.value, eb.value


class Ensemble:
    """Batched FP32-form ensemble through the tsu_ens_* C ABI."""

    def __init__(self, params, switches, device=0):
        n = len(params)
        self.n = n
        self._P = (SimParams * n)(*params)
        self._S = (TsuSwitches * n)(*switches)
        self._h = C.c_void_p()
        _ck(lib().tsu_ens_create(C.byref(self._h), n, C.cast(self._P, C.c_void_p), C.cast(self._S, C.c_void_p),
                                 device), "tsu_ens_create")
        self.members = []
        for i in range(n):
            hs = C.c_void_p()
            _ck(lib().tsu_ens_member(self._h, i, C.byref(hs)), "tsu_ens_member")
            self.members.append(Solver._borrow(hs, self._P[i], self._S[i]))

    def close(self):
        if self._h:
            lib().tsu_ens_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, workloads):
        for s, w in zip(self.members, workloads):
            s.set_state(w.V)
            s.set_mask(w.mask)
            if w.sw.read_files:
                s.set_boundary_series(w.CC, w.tCC)

    def reset(self):
        _ck(lib().tsu_ens_reset(self._h), "tsu_ens_reset")

    def step(self, n):
        _ck(lib().tsu_ens_step(self._h, n), "tsu_ens_step")

    def run_until(self, t_end, max_steps=1 << 40):
        done = C.c_long()
        _ck(lib().tsu_ens_run_until(self._h, t_end, max_steps, C.byref(done)), "tsu_ens_run_until")
        return done.value

    def sync(self):
        _ck(lib().tsu_ens_sync(self._h), "tsu_ens_sync")

    def autotune(self, steps=3):
        buf = C.create_string_buffer(8192)
        _ck(lib().tsu_ens_autotune(self._h, steps, buf, 8192), "tsu_ens_autotune")
        return buf.value.decode()

    def set_config(self, variant, dynamic, ctas=0):
        _ck(lib().tsu_ens_set_config(self._h, variant, dynamic, ctas), "tsu_ens_set_config")

    def config(self):
        v, tx, ty, d, c = (C.c_int() for _ in range(5))
        nt = C.c_long()
        _ck(lib().tsu_ens_get_config(self._h, C.byref(v), C.byref(tx), C.byref(ty), C.byref(d), C.byref(c),
                                     C.byref(nt)), "tsu_ens_get_config")
        return dict(variant=v.value, tile=(tx.value, ty.value), dynamic=bool(d.value), ctas=c.value,
                    ntiles=nt.value)

    def last_ms(self):
        ms = C.c_double()
        _ck(lib().tsu_ens_last_step_ms(self._h, C.byref(ms)), "tsu_ens_last_step_ms")
        return ms.value

    def last_launches(self):
        n = C.c_long()
        _ck(lib().tsu_ens_last_step_launches(self._h, C.byref(n)), "tsu_ens_last_step_launches")
        return n.value


def solver_for(w, device=0):
    """Solver loaded with a workloads.Workload's state, mask and series."""
    s = Solver(w.p, w.sw, device)
    s.set_state(w.V)
    s.set_mask(w.mask)
    if w.sw.read_files:
        s.set_boundary_series(w.CC, w.tCC)
    s.reset()
    return s
