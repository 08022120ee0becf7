#!/usr/bin/env python
"""Benchmark of the TSUNER hot path on B200: cell-steps/s of the time step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload nwave4096|nwave2048|hump512|humps8192|ensembleN|corrector]
                  [--precision fp64|fp32] [--no-cpu-baseline] [--no-config3]

One "step" is one full time step of the scheme (2 RK stages: MUSCL faces,
edge fluxes with bedload, volume update, running extrema, CFL dt) over the
whole grid.  Default workload: the 4096^2 shelf with the west N-wave
(seeded synthetic inputs, no dataset).  The state (671 MB in FP64) is far
larger than the 126 MB L2, so no L2 flush is needed between steps.

--impl ours       the product library (libtsuner_b200.so) through its C ABI.
                  The line's `value` / `e2e` are the FP64 plain form -- the
                  reference's own arithmetic, value-identical to its kernels;
                  the FP32 precision form rides along (`fp32_form`,
                  `fp32_vs_fp64`), and at one GPU the 8192^2 humps
                  configuration runs both forms for a fixed 2000 steps
                  (`config3`: rates, roofline, L-inf / L2 / mass drift).
--impl reference  the reference's own CUDA kernels, unmodified, built by
                  oracle/build_ref.py and driven step by step on the same GPU
                  and inputs (the reference has no CPU implementation of the
                  path); without a GPU or without oracle/_ref it falls back to
                  the oracle port on the host cores.  It never loads the
                  product library.

Multi-GPU (torchrun, one rank per GPU): the grid is split into row slabs,
one per rank (tsuner_b200/slabs.py: a 2-row halo exchange per RK stage by
NCCL send/recv, a MIN all-reduce of the dt per step; strong scaling of the
one grid); --replicas runs one copy of the grid per rank instead (weak
scaling, no data-path collective).  The ensemble workload shares its members
out over the ranks.  The reported time is the max over ranks of the
device-timed region.
"""
import argparse
import ctypes as C
import functools
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s: FP32 fused vs FP64 plain at stated L-inf error; % HBM peak"
# algorithmic DRAM bytes per cell-step of the fused forms, 5 state planes:
# stage 1 reads U^n, writes U*; stage 2 reads U* and U^n, writes U^{n+1}
# (5 x 5 planes x element size), mask read twice (2 x 1 B), hmax/bmin/eta_max
# read-modify-write (3 x 2 x element size)
BYTES_PER_CELL_STEP = {"f64": 5 * 5 * 8 + 2 + 3 * 16, "f32": 5 * 5 * 4 + 2 + 3 * 8}
# the arithmetic both arms compute (the reference's scheme, FP64)
SCHEME = ("FP64; order 2 MUSCL + RK2, HLL-type edge fluctuations with the Ashida-Michiue bedload, Chezy friction, "
          "erosion/deposition, running extrema and the CFL dt every step")
FORM = {0: "fp64 plain form (value-identical to the reference kernels); one fused kernel per RK stage",
        1: "fp32 precision form (FP32 state, FP64 still-water level / wet-dry reconstruction / sums / time); "
           "one fused kernel per RK stage"}
CONFIG3_SIDE = 8192


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload(name):
    from tsuner_b200 import workloads as W
    if name == "nwave4096":
        return W.nwave_shelf(4096, 4096, 5.0), "nwave_shelf 4096x4096 dx=5m (fractal k^-3 shelf, 20% dry, mask, west N-wave 3m/600s, SLR+0.5m)"
    if name == "nwave2048":
        return W.nwave_shelf(2048, 2048, 10.0), "nwave_shelf 2048x2048 dx=10m (profiling case: 168 MB FP64 state > L2)"
    if name == "hump512":
        return W.hump(512, 512, 10.0), "hump 512x512 dx=10m (2m Gaussian hump, noisy 2% slope, walls)"
    if name == "humps8192":
        return W.humps_shelf(8192, 8192, 5.0), "humps_shelf 8192x8192 dx=5m (8 seeded humps, walls)"
    raise SystemExit("unknown workload " + name)


def arm_config(desc, n, world):
    """The config dict both arms print (identical apart from `impl`)."""
    return {"workload": desc, "cells": n, "scheme": SCHEME,
            "l2": "FP64 state %.0f MB > 126 MB L2, no flush needed" % (5 * 8 * n / 1e6),
            "parallelism": "replicas x%d" % world}


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.f = tempfile.TemporaryFile(mode="w+")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.proc:
            return None
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f:
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                mx.append(float(c[2]))
            except ValueError:
                continue
            for n, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


def dist_setup(n, backend=None):
    """One process per GPU (torchrun env).  Replicas only: the process group
    carries the barrier around the timed region and the max over ranks of the
    device time, never data.  backend: "nccl" (default) or "gloo" (CPU
    tests of this plumbing)."""
    if n <= 1 or "RANK" not in os.environ:
        return 0, 1, int(os.environ.get("LOCAL_RANK", 0)), None
    import datetime

    import torch
    import torch.distributed as dist
    backend = backend or os.environ.get("TSU_DIST_BACKEND", "nccl")
    local = int(os.environ.get("LOCAL_RANK", 0))
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist.get_rank(), dist.get_world_size(), local, dist


def _on_gpu(dist):
    return dist.get_backend() == "nccl"


def dist_max(dist, v, local):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=("cuda:%d" % local) if _on_gpu(dist) else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, local):
    if dist is not None:
        import torch
        if _on_gpu(dist):
            dist.barrier(device_ids=[local])
            torch.cuda.synchronize(local)
        else:
            dist.barrier()


def cpu_baseline(max_seconds=20.0):
    """The oracle port (OpenMP C) on this host's cores, on a bounded sample of
    the same workload generator (4096 x 512 strip of the shelf)."""
    import oracle
    from tsuner_b200 import workloads as W
    w = W.nwave_shelf(4096, 512, 5.0)
    r = oracle.OracleRun(w.p, w.sw, w.V, w.mask, w.CC, w.tCC)
    r.run(1)  # first touch of the work arrays
    steps, t0 = 0, time.perf_counter()
    while True:
        r.run(1)
        steps += 1
        el = time.perf_counter() - t0
        if el > max_seconds or steps >= 200:
            break
    return {"value": w.ncells * steps / el / 1e6, "unit": "Mcell-steps/s", "cores": oracle.max_threads(),
            "kind": "port", "sample": "nwave_shelf 4096x512 strip, %d steps (%.1f s) on %d threads"
            % (steps, el, oracle.max_threads())}


def traffic_from_profiles(name):
    """Per-cell-step DRAM bytes of the stage kernels recorded by ncu (profiles/
    traffic.txt): (bytes per cell-step, cells of the capture, capture it came
    from -- another workload's name when the row is scaled per cell)."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) >= 4 and parts[0] == name:
                return float(parts[1]), float(parts[2]), parts[3], float(parts[4]) if len(parts) > 4 else None
    except OSError:
        pass
    return None


def roofline(form, n, steps, ms, tr_key=None):
    hbm, kind = peaks()
    bpc = BYTES_PER_CELL_STEP[form]
    achieved = bpc * n * steps / (ms / 1e3) / 1e9
    r = {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
         "peak_kind": kind, "bytes_per_cell_step": bpc, "traffic": None,
         "note": "algorithmic bytes per cell-step x cells x steps / device time of the stage kernels "
                 "(CUDA events on the solver stream); the kernel is bound by instruction issue, not HBM"}
    tr = traffic_from_profiles(tr_key) if tr_key else None
    if tr is not None:
        # per launch, like `achieved`: bytes per cell-step x cells / 2 stage launches
        r["traffic"] = round(tr[0] * n / 2.0, 0)
        r["traffic_source"] = ("ncu dram__bytes_read+write of this workload" if tr[2] == tr_key else
                               "ncu dram__bytes of the %s capture (%.0f cells) scaled per cell" % (tr[2], tr[1]))
        if tr[3]:
            # the bound that does apply: warp-instruction issue, 4 per clock per SM
            sms, mhz = sm_count_and_max_clock()
            peak_issue = 4.0 * sms * mhz * 1e6
            rate = n * steps / (ms / 1e3)
            r["issue"] = {"warp_inst_per_cell_step": tr[3], "peak_warp_inst_per_s": peak_issue,
                          "frac": round(rate * tr[3] / peak_issue, 4),
                          "source": "ncu smsp__inst_executed of the %s capture per cell-step; peak = 4 warp "
                                    "instructions per clock x %d SMs x %.0f MHz" % (tr[2], sms, mhz)}
    return r


@functools.lru_cache(maxsize=None)
def sm_count_and_max_clock():
    """SMs and maximum SM clock (MHz) of the current device (148, 1965 without one)."""
    try:
        import torch
        if torch.cuda.is_available():
            prop = torch.cuda.get_device_properties(torch.cuda.current_device())
            sms = prop.multi_processor_count
        else:
            sms = 148
    except Exception:
        sms = 148
    mhz = 1965.0
    try:
        out = subprocess.run(["nvidia-smi", "--query-gpu=clocks.max.sm", "--format=csv,noheader,nounits", "-i",
                              str(torch.cuda.current_device())], capture_output=True, text=True, timeout=20)
        mhz = float(out.stdout.strip().splitlines()[0])
    except Exception:
        pass
    return sms, mhz


def form_switches(w, precision):
    from tsuner_b200.abi import make_switches
    sw = w.sw
    return make_switches(order=sw.order, wbc=sw.wbc, bedload=sw.bedload, suspension=sw.suspension,
                         read_files=sw.read_files, bedload_law=sw.bedload_law, precision=precision,
                         grass_ag=sw.grass_ag, eta0=sw.eta0)


def load_solver(T, w, sw, local):
    s = T.Solver(w.p, sw, device=local)
    s.set_state(w.V)
    s.set_mask(w.mask)
    if sw.read_files:
        s.set_boundary_series(w.CC, w.tCC)
    s.reset()
    return s


def pinned(a=None, shape=None, dtype=np.float64):
    """A page-locked host array (a copy of `a`, or empty of `shape`): the e2e
    legs move their inputs and results through pinned host memory."""
    import torch
    src = None if a is None else np.ascontiguousarray(a)
    shp = src.shape if src is not None else shape
    dt = src.dtype if src is not None else np.dtype(dtype)
    t = torch.empty(int(np.prod(shp)) * dt.itemsize, dtype=torch.uint8, pin_memory=True)
    out = t.numpy().view(dt).reshape(shp)  # the array's base chain keeps the tensor alive
    if src is not None:
        out[...] = src
    return out


def run_form(T, w, prec, warmup, steps, local, dist, e2e=True):
    """W warm-up steps, then K device-timed steps (CUDA events on the solver's
    stream, barrier + sync on both sides); then, if e2e, the same K steps end
    to end through the C ABI with host buffers (upload, reset, K steps, state
    and extrema read back).  Returns the state after W + K steps and the
    timings."""
    sw = form_switches(w, prec)
    s = load_solver(T, w, sw, local)
    s.step(warmup)
    s.sync()
    barrier(dist, local)
    with Clocks(local) as clk:
        s.step(steps)
        s.sync()
    out = {"ms": dist_max(dist, s.last_ms(), local), "ms_local": s.last_ms(), "launches": s.last_launches(),
           "clocks": clk.summary(), "V": s.state(), "sums": s.sums() if prec == 1 else None}
    if e2e:
        # inputs and results in pinned host buffers allocated before the timed region
        Vin, Mk = pinned(w.V), pinned(w.mask.astype(np.int32))
        CCp, tCp = (pinned(w.CC), pinned(w.tCC)) if sw.read_files else (None, None)
        Vout = pinned(shape=w.V.shape)
        ext = [pinned(shape=w.V.shape[1:]) for _ in range(3)]
        L = T.lib()
        barrier(dist, local)
        t0 = time.perf_counter()
        s.set_state(Vin)
        s.set_mask(Mk)
        if sw.read_files:
            s.set_boundary_series(CCp, tCp)
        s.reset()
        s.step(steps)
        rc = L.tsu_get_state(s._h, Vout.ctypes.data_as(C.c_void_p))
        rc |= L.tsu_get_extrema(s._h, *[e.ctypes.data_as(C.c_void_p) for e in ext])
        out["e2e_s"] = dist_max(dist, time.perf_counter() - t0, local)
        assert rc == 0 and np.isfinite(Vout).all()
    s.close()
    return out


def e2e_line(world, n, steps, e2e_s, w):
    h2d = 5 * 8 * n + 4 * n + (w.CC.nbytes + w.tCC.nbytes if w.sw.read_files else 0)
    d2h = 5 * 8 * n + 3 * 8 * n
    return {"value": round(world * n * steps / e2e_s / 1e6, 3), "unit": "Mcell-steps/s",
            "h2d_bytes_per_step": int(h2d / steps), "d2h_bytes_per_step": int(d2h / steps),
            "what": "tsu_set_state/mask/series + tsu_reset + tsu_step(K) + tsu_get_state/extrema, pinned host "
                    "buffers (copies inside the timed region, amortised over the K = %d steps)" % steps}


def depth_errors(V32, V64, eps_h):
    wet = V64[0] > eps_h
    dh = V32[0] - V64[0]
    m32, m64 = float(V32[0].sum()), float(V64[0].sum())
    return {"linf_depth_m": float(np.abs(dh).max()),
            "l2_depth_m": float(np.sqrt(np.mean(dh[wet] ** 2))) if wet.any() else 0.0,
            "linf_qx": float(np.abs(V32[1] - V64[1]).max()),
            "linf_bed_m": float(np.abs(V32[3] - V64[3]).max()),
            "mass_drift_rel": (m32 - m64) / m64 if m64 else None}


def run_config3(a, T, local):
    """Config 3: humps_shelf 8192^2 (67.1 M cells), both forms for a fixed
    number of steps from the same initial state (5 untimed, the rest timed),
    then the FP32 form's depth error and mass drift against the FP64 form."""
    from tsuner_b200 import workloads as W
    w = W.humps_shelf(CONFIG3_SIDE, CONFIG3_SIDE, 5.0)
    n = w.ncells
    total, warm = a.config3_steps, 5
    timed = total - warm
    m0 = float(w.V[0].sum())
    r = {}
    for prec in (1, 0):
        r[prec] = run_form(T, w, prec, warm, timed, local, None, e2e=False)
    V32, V64 = r[1]["V"], r[0]["V"]
    err = depth_errors(V32, V64, w.p.epsilon_h)
    err["steps"] = total
    err["mass_change_rel"] = {"fp32": (float(V32[0].sum()) - m0) / m0, "fp64": (float(V64[0].sum()) - m0) / m0}
    err["bound_linf_depth_m"] = 1e-4
    out = {"workload": "humps_shelf %dx%d dx=5m (8 seeded humps 0.5-4 m / sigma 200-2000 m, fractal shelf, "
                       "harbour mask, walls), %d steps (%d warm-up + %d timed)" % (CONFIG3_SIDE, CONFIG3_SIDE, total,
                                                                              warm, timed),
           "cells": n}
    for prec, key, form in ((1, "fp32", "f32"), (0, "fp64", "f64")):
        out[key] = {"value": round(n * timed / (r[prec]["ms"] / 1e3) / 1e6, 3), "unit": "Mcell-steps/s",
                    "ms_per_step": round(r[prec]["ms"] / timed, 4),
                    "roofline": roofline(form, n, timed, r[prec]["ms"],
                                         ("stage32_" if prec else "stage64_") + "humps8192"),
                    "clocks": r[prec]["clocks"], "gpu_launches": r[prec]["launches"]}
    out["fp32_over_fp64"] = round(r[0]["ms"] / r[1]["ms"], 3)
    out["fp32_vs_fp64"] = err
    return out


def shard_members(ws, world, rank):
    """Members of this rank: the largest first, each to the least loaded rank
    (cells), so that the ranks' shares of the cell count stay close."""
    load = [0] * world
    mine = []
    for i in sorted(range(len(ws)), key=lambda i: -ws[i].ncells):
        r = min(range(world), key=lambda q: load[q])
        load[r] += ws[i].ncells
        if r == rank:
            mine.append(ws[i])
    return mine


def run_decomposed(a, rank, world, local, dist):
    """One grid split into row slabs, one per rank (tsuner_b200/slabs.py):
    per RK stage a 2-row halo exchange by NCCL send/recv, per step a MIN
    all-reduce of the dt; strong scaling of the single grid.  FP64 plain form
    (the reference's arithmetic).  Device time: CUDA events on the stream the
    slabs and their messages use, max over ranks."""
    import torch

    from tsuner_b200 import slabs as S
    w, desc = workload(a.workload)
    n = w.ncells
    sw = form_switches(w, 0)
    g = S.SlabGroup(w.p, sw, dist=dist, device=local)
    g.load(w.V, w.mask, w.CC, w.tCC)
    g.reset()
    g.step(a.warmup)
    g.sync()
    barrier(dist, local)
    st = torch.cuda.current_stream(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        e0.record(st)
        g.step(a.steps)
        e1.record(st)
        g.sync()
    ms = dist_max(dist, e0.elapsed_time(e1), local)
    barrier(dist, local)
    t0 = time.perf_counter()
    g.load(w.V, w.mask, w.CC, w.tCC)
    g.reset()
    g.step(a.steps)
    parts = g.local_state()
    g.local_extrema()
    e2e_s = dist_max(dist, time.perf_counter() - t0, local)
    g.close()
    assert all(np.isfinite(v).all() for _, v in parts.values())
    if rank != 0:
        return None
    cfg = arm_config(desc, n, world)
    cfg["parallelism"] = ("row slabs x%d (2-row halo of the 5 state planes per RK stage by NCCL send/recv into "
                          "local buffers, 8-byte MIN all-reduce of dt per step)" % world)
    return {
        "metric": METRIC, "value": round(n * a.steps / (ms / 1e3) / 1e6, 3), "unit": "Mcell-steps/s",
        "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 4),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generators, no dataset)", "config": cfg, "form": FORM[0],
        "roofline": roofline("f64", n, a.steps, ms, "stage64_" + a.workload),
        "gpu_launches": 2 * a.steps,
        "e2e": {"value": round(n * a.steps / e2e_s / 1e6, 3), "unit": "Mcell-steps/s",
                "h2d_bytes_per_step": int((5 * 8 * n + 4 * n + w.CC.nbytes + w.tCC.nbytes) / a.steps),
                "d2h_bytes_per_step": int((5 * 8 * n + 3 * 8 * n) / a.steps),
                "what": "every rank: its slab's upload, reset, K steps with the exchanges, read-back; max over ranks"},
        "clocks": clk.summary(),
    }


def run_ensemble(a, rank, world, local, dist):
    """Config 4: batched FP32 ensemble; value = sum(cells) x steps / time.
    With several GPUs the members are shared out among the ranks (no
    exchange between members); the time is the max over ranks."""
    import tsuner_b200 as T
    from tsuner_b200 import workloads as W
    nmem = int(a.workload[len("ensemble"):] or 256)
    ws_all = W.ensemble(nmembers=nmem)
    ws = shard_members(ws_all, world, rank) if world > 1 else ws_all
    cells = sum(w.ncells for w in ws_all)
    e = T.Ensemble([w.p for w in ws], [w.sw for w in ws], device=local)
    e.load(ws)
    e.reset()
    report = e.autotune(steps=2)
    cfg = e.config()
    e.step(a.warmup)
    e.sync()
    barrier(dist, local)
    with Clocks(local) as clk:
        e.step(a.steps)
        e.sync()
    ms = e.last_ms()
    launches = e.last_launches()
    ms_max = dist_max(dist, ms, local)
    # the same members stepped one after the other with the single-grid kernels
    ms_seq = 0.0
    for s in e.members:
        s.step(a.steps)
        s.sync()
        ms_seq += s.last_ms()
    # end to end: upload every member, reset, K steps, read every member back
    barrier(dist, local)
    t0 = time.perf_counter()
    e.load(ws)
    e.reset()
    e.step(a.steps)
    e.sync()
    finite = all(np.isfinite(s.state()).all() for s in e.members)
    e2e_s = dist_max(dist, time.perf_counter() - t0, local)
    e.close()
    assert finite
    if rank != 0:
        return None
    hbm, kind = peaks()
    bpc = BYTES_PER_CELL_STEP["f32"]
    cells_here = sum(w.ncells for w in ws)  # this rank's share (rank 0)
    achieved = bpc * cells_here * a.steps / (ms / 1e3) / 1e9
    h2d = sum(5 * 8 * w.ncells + 4 * w.ncells + w.CC.nbytes + w.tCC.nbytes for w in ws)
    d2h = sum(5 * 8 * w.ncells for w in ws)
    return {
        "metric": METRIC, "value": round(cells * a.steps / (ms_max / 1e3) / 1e6, 3),
        "unit": "Mcell-steps/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": round(ms_max / a.steps, 4), "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators, no dataset)",
        "config": {"workload": "ensemble of %d members, square sides log-uniform in [256, 2048] (seed 4), "
                               "own shelf bathymetry / mask / west N-wave each" % nmem,
                   "cells": cells, "form": "fp32 precision form, one persistent launch per RK stage over all "
                                            "members, per-member dt, CUDA graph",
                   "tile": cfg, "autotune": report.strip().splitlines(),
                   "parallelism": ("members shared out over %d ranks (largest first to the least loaded; "
                                   "no exchange)" % world) if world > 1 else "single GPU"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4), "peak_kind": kind, "bytes_per_cell_step": bpc,
                     "traffic": None},
        "members_one_by_one": {"value": round(cells_here * a.steps / (ms_seq / 1e3) / 1e6, 3), "unit": "Mcell-steps/s",
                               "ms_per_step": round(ms_seq / a.steps, 4)},
        "gpu_launches": launches,
        "e2e": {"value": round(cells * a.steps / e2e_s / 1e6, 3), "unit": "Mcell-steps/s",
                "h2d_bytes_per_step": int(h2d / a.steps), "d2h_bytes_per_step": int(d2h / a.steps),
                "what": "upload all members + reset + K steps + read all members back, host buffers"},
        "clocks": clk.summary(),
    }


def run_corrector(a, rank, world, local, dist):
    """Learned corrector (reduced config 5): FP32 coarse solves (factor 4)
    lifted to fine maximum-depth / bed-change maps; the pairs come from the
    solver (FP32 ensembles), the held-out truth from the FP64 plain form.
    Reports held-out error with and without the corrector, training time and
    the tensor-core convolution's TFLOP/s.  Replicas only (each rank runs the
    whole pipeline)."""
    from tsuner_b200 import corrector as K
    n, f, t_end = a.corr_fine, 4, a.corr_tend
    site = K.make_site(n=n, factor=f, dx=a.corr_dx)
    train_src = K.make_sources(a.corr_train, seed=11)
    test_src = K.make_sources(a.corr_test, seed=12)
    t0 = time.perf_counter()
    fine_train = K.solve_fp32(site.H, site.mask, site.dx, site.slr, train_src, t_end)
    t_fine = time.perf_counter() - t0
    coarse_train = K.coarse_inputs(site, train_src, t_end)
    coarse_test = K.coarse_inputs(site, test_src, t_end)
    t0 = time.perf_counter()
    truth = K.solve_fp64(site.H, site.mask, site.dx, site.slr, test_src, t_end)
    t_truth = time.perf_counter() - t0
    c = K.Corrector(n, n, f, max_batch=8, device=local)
    c.set_site(site.H)
    c.set_options(a.corr_wbig, a.corr_clip, a.corr_envelope)
    c.add_samples(coarse_train, fine_train)
    c.add_samples(coarse_test, truth)
    # step-wise decay: half the steps at 1e-3, a quarter at 3e-4, a quarter at 1e-4
    # (Adam moments carry over between the calls)
    losses, train_ms, convs = [], 0.0, 0
    phases = [(a.corr_iters // 2, 1e-3), (a.corr_iters // 4, 3e-4), (a.corr_iters - a.corr_iters // 2 - a.corr_iters // 4, 1e-4)]
    for k, (it, lr) in enumerate(phases):
        if it > 0:
            losses.append(c.train(len(train_src), it, batch=8, lr=lr, seed=1 + k))
            ms_k, n_k = c.last_train()
            train_ms += ms_k
            convs += n_k
    loss = np.concatenate(losses)
    oh, ob, bh, bb = c.predict(len(train_src), len(test_src))
    with Clocks(local) as clk:
        ms_conv, tflops = c.bench_conv(8, max(a.steps, 5))
    c.close()
    region = (truth[:, 0] > 0) | (oh != 0) | (bh != 0)  # one denominator for both RMSEs
    e_with = K.errors((oh, ob), truth, region)
    e_without = K.errors((bh, bb), truth, region)
    if rank != 0:
        return None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peak, kind = float(json.load(fh)["bf16_tflops"]), "measured (burst)"
    except Exception:
        peak, kind = 1590.0, "fallback"
    return {
        "metric": "corrector: held-out fine-map error with/without; tensor-core conv TFLOP/s", "value": round(tflops, 1),
        "unit": "TFLOP/s", "n_gpus": world, "steps": max(a.steps, 5), "warmup": 3,
        "ms_per_step": round(ms_conv, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16 (fp32 accumulate)", "data": "synthetic (seeded site and sources, solver-generated pairs)",
        "config": {"workload": "corrector: fine %dx%d dx=%.0fm <- coarse %dx%d, %d train pairs (FP32 ensembles), "
                               "%d held-out sources compared against the FP64 plain solve, t_end %.0f s"
                               % (n, n, site.dx, n // f, n // f, len(train_src), len(test_src), t_end),
                   "network": "6 x conv3x3 32 ch, BF16 weights/activations, FP32 accumulate (tcgen05, TMEM)",
                   "train": {"iters": a.corr_iters, "batch": 8, "lr": "1e-3 / 3e-4 / 1e-4 (1/2, 1/4, 1/4 of the steps)",
                             "large_residual_weight": a.corr_wbig, "clip_depth": bool(a.corr_clip),
                             "envelope": a.corr_envelope,
                             "ms": round(train_ms, 1),
                             "convs": convs, "loss_first": float(loss[:5].mean()),
                             "loss_last": float(loss[-10:].mean())},
                   "solve_seconds": {"fine_fp32_train": round(t_fine, 2), "fine_fp64_heldout": round(t_truth, 2)},
                   "parallelism": "replicas x%d" % world},
        "errors": {"with_corrector": e_with, "interpolation_only": e_without},
        "roofline": {"bound": "tensor", "achieved": round(tflops, 1), "peak": peak, "unit": "TFLOP/s",
                     "frac": round(tflops / peak, 4), "peak_kind": kind, "traffic": None,
                     "note": "2 x pixels x 288 x 32 FLOPs per 3x3 convolution, 8 images per launch"},
        "gpu_launches": max(a.steps, 5),
        "clocks": clk.summary(),
    }


def run_ours(a, rank, world, local, dist):
    import tsuner_b200 as T
    if a.workload.startswith("ensemble"):
        return run_ensemble(a, rank, world, local, dist)
    if a.workload == "corrector":
        return run_corrector(a, rank, world, local, dist)
    if world > 1 and not a.replicas:
        return run_decomposed(a, rank, world, local, dist)
    w, desc = workload(a.workload)
    n = w.ncells
    prim = 1 if a.precision == "fp32" else 0
    other = 1 - prim
    # ---- primary form: device-timed with inputs resident in HBM, then end to end
    P = run_form(T, w, prim, a.warmup, a.steps, local, dist)
    # ---- the other form on the same workload and step count (rate, e2e, error)
    O = None if a.no_other else run_form(T, w, other, a.warmup, a.steps, local, dist)
    C3 = None
    if world == 1 and not a.no_config3 and a.workload == "nwave4096":
        C3 = run_config3(a, T, local)
    if rank != 0:
        return None
    dtype = "f32" if prim == 1 else "f64"
    line = {
        "metric": METRIC, "value": round(world * n * a.steps / (P["ms"] / 1e3) / 1e6, 3), "unit": "Mcell-steps/s",
        "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(P["ms"] / a.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
        "data": "synthetic (seeded generators, no dataset)",
        "config": arm_config(desc, n, world),
        "form": FORM[prim],
        "roofline": roofline(dtype, n, a.steps, P["ms_local"], ("stage32_" if prim else "stage64_") + a.workload),
        "gpu_launches": P["launches"],
        "e2e": e2e_line(world, n, a.steps, P["e2e_s"], w),
        "clocks": P["clocks"],
    }
    if O is not None:
        key = "fp32_form" if other == 1 else "fp64_plain"
        oform = "f32" if other == 1 else "f64"
        line[key] = {"value": round(world * n * a.steps / (O["ms"] / 1e3) / 1e6, 3), "unit": "Mcell-steps/s",
                     "ms_per_step": round(O["ms"] / a.steps, 4), "form": FORM[other],
                     "roofline": roofline(oform, n, a.steps, O["ms_local"],
                                          ("stage32_" if other else "stage64_") + a.workload),
                     "e2e": e2e_line(world, n, a.steps, O["e2e_s"], w), "gpu_launches": O["launches"],
                     "clocks": O["clocks"]}
        V32, V64 = (P["V"], O["V"]) if prim == 1 else (O["V"], P["V"])
        err = depth_errors(V32, V64, w.p.epsilon_h)
        err["steps"] = a.warmup + a.steps
        ms32, ms64 = (P["ms"], O["ms"]) if prim == 1 else (O["ms"], P["ms"])
        err["speedup"] = round(ms64 / ms32, 3)
        line["fp32_vs_fp64"] = err
    if C3 is not None:
        line["config3"] = C3
    if world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    return line


def run_reference(a, rank, world, local, dist):
    """The reference's own CUDA kernels (oracle/_ref/default: the makefile
    recipe build of its unmodified GPU sources) on the same workload, one
    replica per rank; without a GPU or without the build, the oracle port on
    rank 0's host cores.  The product library is never loaded here."""
    import oracle
    w, desc = workload(a.workload)
    n = w.ncells
    if n > 53687091:  # GPU/main_TSUNER.cu:60-90: int size arithmetic overflows above this
        if rank == 0:
            return {"impl": "reference", "unavailable": "the reference cannot allocate a %dx%d grid (int overflow in "
                                                         "its size arithmetic, GPU/main_TSUNER.cu:60-90)"
                                                         % (w.p.npx, w.p.npy)}
        return None
    gpu_ok = oracle.ref_gpu_count("default") > local
    if gpu_ok:
        CC, tCC = (w.CC, w.tCC) if w.sw.read_files else oracle_expired(w)
        oracle.ref_run("default", w.p, w.V, w.mask, CC, tCC, a.warmup, device=local)
        # the same pinned host buffers as the product's e2e leg, filled before the timed call
        work, Mk, CCp, tCp = pinned(w.V), pinned(w.mask.astype(np.int32)), pinned(CC), pinned(tCC)
        ext = [pinned(shape=w.V.shape[1:]) for _ in range(3)]
        barrier(dist, local)
        with Clocks(local) as clk:
            t0 = time.perf_counter()
            r = oracle.ref_run("default", w.p, None, Mk, CCp, tCp, a.steps, device=local, work=work, ext=ext)
            wall = time.perf_counter() - t0
        ms = dist_max(dist, r["ms"], local)
        wall = dist_max(dist, wall, local)
        if rank != 0:
            return None
        value = world * n * a.steps / (ms / 1e3) / 1e6
        return {"metric": METRIC, "value": round(value, 3), "unit": "Mcell-steps/s", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 4),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generators, no dataset)", "impl": "reference",
                "reference_kind": "reference CUDA build (unmodified GPU/*.cu kernels, -O2 -fmad=false -rdc -dlto, "
                                  "sm_100a), stepped by oracle/ref_build/ref_harness.cu",
                "config": arm_config(desc, n, world),
                "e2e": {"value": round(world * n * a.steps / wall / 1e6, 3), "unit": "Mcell-steps/s",
                        "h2d_bytes_per_step": int((5 * 8 * n + 4 * n + (CC.nbytes + tCC.nbytes)) / a.steps),
                        "d2h_bytes_per_step": int((5 * 8 * n + 3 * 8 * n) / a.steps),
                        "what": "whole harness call: allocation, upload, K steps, download, pinned host buffers"},
                "clocks": clk.summary()}
    if rank != 0:
        return None
    cb = cpu_baseline()
    return {"metric": METRIC, "value": cb["value"], "unit": "Mcell-steps/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference", "config": arm_config(desc, n, world),
            "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "Mcell-steps/s",
                                        "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def oracle_expired(w):
    from tsuner_b200 import workloads as W
    return W.expired_series(w.p.npx, w.p.npy)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="nwave4096")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"],
                    help="form of the line's value / e2e (the other form is reported beside it)")
    ap.add_argument("--no-other", "--no-fp64", dest="no_other", action="store_true",
                    help="skip the other form's run")
    ap.add_argument("--no-config3", action="store_true", help="skip the 8192^2 configuration")
    ap.add_argument("--replicas", action="store_true",
                    help="with several GPUs: one copy of the grid per rank instead of one grid in row slabs")
    ap.add_argument("--config3-steps", type=int, default=2000, help="steps of the 8192^2 configuration")
    ap.add_argument("--corr-fine", type=int, default=512, help="corrector: fine grid side")
    ap.add_argument("--corr-train", type=int, default=128, help="corrector: training pairs")
    ap.add_argument("--corr-test", type=int, default=16, help="corrector: held-out sources")
    ap.add_argument("--corr-iters", type=int, default=400, help="corrector: Adam steps")
    ap.add_argument("--corr-tend", type=float, default=600.0, help="corrector: simulated seconds per source")
    ap.add_argument("--corr-dx", type=float, default=10.0, help="corrector: fine cell size (m)")
    ap.add_argument("--corr-wbig", type=float, default=16.0,
                    help="corrector: loss weight 1 + w t^2 on large maximum-depth residuals")
    ap.add_argument("--corr-clip", type=int, default=1, choices=[0, 1],
                    help="corrector: clip the corrected maximum depth at 0")
    ap.add_argument("--corr-envelope", type=float, default=1.0,
                    help="corrector: clamp residuals to k x the training pairs' per-pixel envelope (0 = off)")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)
    a.config3_steps = max(a.config3_steps, 10)
    rank, world, local, dist = dist_setup(a.gpus)
    try:
        if a.impl == "reference":
            line = run_reference(a, rank, world, local, dist)
        else:
            line = run_ours(a, rank, world, local, dist)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
