#!/usr/bin/env python
"""Benchmark of the TSUNER hot path on B200: cell-steps/s of the time step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload nwave4096|nwave2048|hump512|humps8192|ensembleN|corrector]
                  [--no-cpu-baseline]

One "step" is one full time step of the scheme (2 RK stages: MUSCL faces,
edge fluxes with bedload, volume update, running extrema, CFL dt) over the
whole grid.  Default workload: the 4096^2 shelf with the west N-wave
(seeded synthetic inputs, no dataset).  The state (671 MB in FP64) is far
larger than the 126 MB L2, so no L2 flush is needed between steps.

--impl ours       the product library (libtsuner_b200.so) through its C ABI
--impl reference  the reference's own CUDA kernels, unmodified, built by
                  oracle/build_ref.py and driven step by step on the same GPU
                  and inputs (the reference has no CPU implementation of the
                  path); without a GPU or without oracle/_ref it falls back to
                  the oracle port on the host cores.

Multi-GPU (torchrun, one rank per GPU): every rank advances its own replica
(weak scaling, no data-path collective); the reported time is the max over
ranks of the device-timed region.
"""
import argparse
import ctypes as C
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
    """Per-launch DRAM bytes of the stage kernels recorded by ncu (profiles/)."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) >= 3 and parts[0] == name:
                return float(parts[1]), float(parts[2])  # bytes per cell-step, cells of the capture
    except OSError:
        pass
    return None


def timed_form(T, w, sw, a, local, dist):
    """W warm-up steps, then K device-timed steps (CUDA events on the solver's
    stream, barrier + sync on both sides).  Returns the solver (state after
    W + K steps) and the timing."""
    s = T.Solver(w.p, sw, device=local)
    s.set_state(w.V)
    s.set_mask(w.mask)
    if sw.read_files:
        s.set_boundary_series(w.CC, w.tCC)
    s.reset()
    s.step(a.warmup)
    s.sync()
    barrier(dist, local)
    with Clocks(local) as clk:
        s.step(a.steps)
        s.sync()
    ms = s.last_ms()
    return s, ms, s.last_launches(), clk.summary()


def form_switches(w, precision):
    from tsuner_b200.abi import make_switches
    sw = w.sw
    return make_switches(order=sw.order, wbc=sw.wbc, bedload=sw.bedload, suspension=sw.suspension,
                         read_files=sw.read_files, bedload_law=sw.bedload_law, precision=precision,
                         grass_ag=sw.grass_ag, eta0=sw.eta0)


def run_ensemble(a, rank, world, local, dist):
    """Config 4: batched FP32 ensemble; value = sum(cells) x steps / time."""
    import tsuner_b200 as T
    from tsuner_b200 import workloads as W
    nmem = int(a.workload[len("ensemble"):] or 256)
    ws = W.ensemble(nmembers=nmem)
    cells = sum(w.ncells for w in ws)
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
    achieved = bpc * cells * a.steps / (ms / 1e3) / 1e9
    h2d = sum(5 * 8 * w.ncells + 4 * w.ncells + w.CC.nbytes + w.tCC.nbytes for w in ws)
    d2h = sum(5 * 8 * w.ncells for w in ws)
    return {
        "metric": METRIC, "value": round(world * cells * a.steps / (ms_max / 1e3) / 1e6, 3),
        "unit": "Mcell-steps/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": round(ms_max / a.steps, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators, no dataset)",
        "config": {"workload": "ensemble of %d members, square sides log-uniform in [256, 2048] (seed 4), "
                               "own shelf bathymetry / mask / west N-wave each" % nmem,
                   "cells": cells, "form": "fp32 precision form, one persistent launch per RK stage over all "
                                            "members, per-member dt, CUDA graph",
                   "tile": cfg, "autotune": report.strip().splitlines(),
                   "parallelism": "replicas x%d" % world},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4), "peak_kind": kind, "bytes_per_cell_step": bpc,
                     "traffic": None},
        "members_one_by_one": {"value": round(cells * a.steps / (ms_seq / 1e3) / 1e6, 3), "unit": "Mcell-steps/s",
                               "ms_per_step": round(ms_seq / a.steps, 4)},
        "gpu_launches": launches,
        "e2e": {"value": round(world * cells * a.steps / e2e_s / 1e6, 3), "unit": "Mcell-steps/s",
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
    site = K.make_site(n=n, factor=f)
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
    e_with = K.errors((oh, ob), truth)
    e_without = K.errors((bh, bb), truth)
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
    w, desc = workload(a.workload)
    n = w.ncells
    prim = 1 if a.precision == "fp32" else 0
    # ---- primary form, device-timed with inputs resident in HBM
    s, ms, launches, clocks = timed_form(T, w, form_switches(w, prim), a, local, dist)
    ms_max = dist_max(dist, ms, local)
    V_prim = s.state()
    sums = s.sums() if prim == 1 else None
    # ---- end to end through the C ABI with host buffers
    barrier(dist, local)
    t0 = time.perf_counter()
    s.set_state(w.V)
    s.set_mask(w.mask)
    if w.sw.read_files:
        s.set_boundary_series(w.CC, w.tCC)
    s.reset()
    s.step(a.steps)
    Vout = s.state()
    s.extrema()
    e2e_s = dist_max(dist, time.perf_counter() - t0, local)
    s.close()
    assert np.isfinite(Vout).all()
    # ---- the other form on the same workload and step count (rate + error)
    other = None
    if prim == 1 and not a.no_fp64:
        s64, ms64, _, _ = timed_form(T, w, form_switches(w, 0), a, local, dist)
        ms64 = dist_max(dist, ms64, local)
        V64 = s64.state()
        s64.close()
        wet = V64[0] > w.p.epsilon_h
        dh = V_prim[0] - V64[0]
        m64 = float(V64[0].sum())
        hbm64, kind64 = peaks()
        ach64 = BYTES_PER_CELL_STEP["f64"] * n * a.steps / (ms64 / 1e3) / 1e9
        other = {"fp64_plain": {"value": round(world * n * a.steps / (ms64 / 1e3) / 1e6, 3),
                                "unit": "Mcell-steps/s", "ms_per_step": round(ms64 / a.steps, 4),
                                "roofline": {"bound": "hbm", "achieved": round(ach64, 1), "peak": hbm64,
                                             "unit": "GB/s", "frac": round(ach64 / hbm64, 4), "peak_kind": kind64,
                                             "bytes_per_cell_step": BYTES_PER_CELL_STEP["f64"]}},
                 "fp32_vs_fp64": {"steps": a.warmup + a.steps,
                                  "linf_depth_m": float(np.abs(dh).max()),
                                  "l2_depth_m": float(np.sqrt(np.mean(dh[wet] ** 2))) if wet.any() else 0.0,
                                  "linf_qx": float(np.abs(V_prim[1] - V64[1]).max()),
                                  "mass_drift_rel": (sums[0] - m64) / m64 if sums else None,
                                  "speedup": round(ms64 / ms, 3)}}
    h2d = 5 * 8 * n + 4 * n + (w.CC.nbytes + w.tCC.nbytes if w.sw.read_files else 0)
    d2h = 5 * 8 * n + 3 * 8 * n
    if rank != 0:
        return None
    value = world * n * a.steps / (ms_max / 1e3) / 1e6
    hbm, kind = peaks()
    dtype = "f32" if prim == 1 else "f64"
    bpc = BYTES_PER_CELL_STEP[dtype]
    achieved = bpc * n * a.steps / (ms / 1e3) / 1e9
    tr = traffic_from_profiles(("stage32_" if prim else "stage64_") + a.workload)
    form = ("fp32 precision form (FP32 state, FP64 still-water level / wet-dry reconstruction / sums / time)"
            if prim else "fp64 plain form (value-identical to the reference kernels)")
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Mcell-steps/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms_max / a.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
        "data": "synthetic (seeded generators, no dataset)",
        "config": {"workload": desc, "form": form + "; one fused kernel per RK stage",
                   "cells": n, "l2": "state %.0f MB > 126 MB L2, no flush needed" % (5 * (4 if prim else 8) * n / 1e6),
                   "parallelism": "replicas x%d" % world},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4), "peak_kind": kind,
                     "bytes_per_cell_step": bpc,
                     "traffic": None if tr is None else round(tr[0] * n / 2.0, 0),
                     "note": "algorithmic bytes per cell-step x cells x steps / device time of the stage kernels"},
        "gpu_launches": launches,
        "e2e": {"value": round(world * n * a.steps / e2e_s / 1e6, 3), "unit": "Mcell-steps/s",
                "h2d_bytes_per_step": int(h2d / a.steps), "d2h_bytes_per_step": int(d2h / a.steps),
                "what": "tsu_set_state/mask/series + tsu_reset + tsu_step(K) + tsu_get_state/extrema, host buffers"},
        "clocks": clocks,
    }
    if other:
        line.update(other)
    if world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    return line


def run_reference(a, rank, world, local, dist):
    if rank != 0:
        return None
    import oracle
    w, desc = workload(a.workload)
    n = w.ncells
    gpu_ok = False
    try:
        import tsuner_b200 as T
        gpu_ok = T.lib().checkCUDAsupport(local) == 0
    except Exception:
        gpu_ok = False
    if gpu_ok and oracle.ref_available("default"):
        CC, tCC = (w.CC, w.tCC) if w.sw.read_files else oracle_expired(w)
        oracle.ref_run("default", w.p, w.V, w.mask, CC, tCC, a.warmup, device=local)
        with Clocks(local) as clk:
            t0 = time.perf_counter()
            r = oracle.ref_run("default", w.p, w.V, w.mask, CC, tCC, a.steps, device=local)
            wall = time.perf_counter() - t0
        value = n * a.steps / (r["ms"] / 1e3) / 1e6
        return {"metric": METRIC, "value": round(value, 3), "unit": "Mcell-steps/s", "n_gpus": 1,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(r["ms"] / a.steps, 4),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generators, no dataset)", "impl": "reference",
                "reference_kind": "reference CUDA build (unmodified GPU/*.cu kernels, -O2 -fmad=false -rdc -dlto, sm_100a)",
                "config": {"workload": desc, "cells": n, "parallelism": "single GPU"},
                "e2e": {"value": round(n * a.steps / wall / 1e6, 3), "unit": "Mcell-steps/s",
                        "h2d_bytes_per_step": int((5 * 8 * n + 4 * n) / a.steps),
                        "d2h_bytes_per_step": int((5 * 8 * n + 3 * 8 * n) / a.steps),
                        "what": "whole harness call: allocation, upload, K steps, download"},
                "clocks": clk.summary()}
    cb = cpu_baseline()
    return {"metric": METRIC, "value": cb["value"], "unit": "Mcell-steps/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference", "config": {"workload": desc},
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
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--corr-fine", type=int, default=512, help="corrector: fine grid side")
    ap.add_argument("--corr-train", type=int, default=128, help="corrector: training pairs")
    ap.add_argument("--corr-test", type=int, default=16, help="corrector: held-out sources")
    ap.add_argument("--corr-iters", type=int, default=400, help="corrector: Adam steps")
    ap.add_argument("--corr-tend", type=float, default=600.0, help="corrector: simulated seconds per source")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)
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
