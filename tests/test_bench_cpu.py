"""CPU: the bookkeeping of bench.py's JSON line -- the algorithmic bytes,
the HBM and instruction-issue roofline arithmetic, the ncu table it reads
(profiles/traffic.txt), the config both arms print and the sharing of
ensemble members among ranks.  No kernel is launched."""
import os

import pytest

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_algorithmic_bytes_per_cell_step():
    # 5 planes x (U^n read, U* write, U* read, U^n read, U^{n+1} write) + mask twice + 3 extrema read and written
    assert bench.BYTES_PER_CELL_STEP["f64"] == 5 * 5 * 8 + 2 + 3 * 2 * 8 == 250
    assert bench.BYTES_PER_CELL_STEP["f32"] == 5 * 5 * 4 + 2 + 3 * 2 * 4 == 126


def test_every_traffic_row_is_read_and_scaled_rows_name_their_capture():
    rows = [l.split() for l in open(os.path.join(ROOT, "profiles", "traffic.txt")) if l.strip() and l[0] != "#"]
    assert rows
    for name, bpc, cells, capture, winst in rows:
        tr = bench.traffic_from_profiles(name)
        assert tr == (float(bpc), float(cells), capture, float(winst))
        form = "f64" if name.startswith("stage64") else "f32"
        # measured DRAM traffic at or below the algorithmic bytes: no re-reads
        assert 0 < float(bpc) <= bench.BYTES_PER_CELL_STEP[form]
        assert capture.split("_")[0] == name.split("_")[0]
    assert bench.traffic_from_profiles("no_such_kernel") is None


def test_roofline_arithmetic():
    n, steps, ms = 16777216, 20, 120.0
    r = bench.roofline("f64", n, steps, ms, "stage64_nwave4096")
    hbm, _ = bench.peaks()
    achieved = 250 * n * steps / (ms / 1e3) / 1e9
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["peak"] == hbm
    assert r["achieved"] == pytest.approx(achieved, abs=0.1)
    assert r["frac"] == pytest.approx(achieved / hbm, abs=1e-4)
    bpc, _, capture, winst = bench.traffic_from_profiles("stage64_nwave4096")
    assert r["traffic"] == pytest.approx(bpc * n / 2, rel=1e-9)  # per launch, two launches a step
    assert capture in r["traffic_source"]
    sms, mhz = bench.sm_count_and_max_clock()
    rate = n * steps / (ms / 1e3)
    assert r["issue"]["frac"] == pytest.approx(rate * winst / (4.0 * sms * mhz * 1e6), abs=1e-4)
    assert bench.roofline("f32", n, steps, ms)["traffic"] is None  # no capture named: no traffic figure


def test_both_arms_print_the_same_config():
    a = bench.arm_config("nwave_shelf 4096x4096", 16777216, 1)
    b = bench.arm_config("nwave_shelf 4096x4096", 16777216, 1)
    assert a == b and a["parallelism"] == "replicas x1" and a["cells"] == 16777216


class _M:
    def __init__(self, n):
        self.ncells = n


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_ensemble_members_are_shared_out_once_and_evenly(world):
    sizes = [256 ** 2, 2048 ** 2, 300 ** 2, 1024 ** 2, 777 ** 2, 1500 ** 2, 512 ** 2, 2000 ** 2, 400 ** 2]
    ws = [_M(n) for n in sizes]
    parts = [bench.shard_members(ws, world, r) for r in range(world)]
    got = sorted(id(m) for p in parts for m in p)
    assert got == sorted(id(m) for m in ws)  # every member on exactly one rank
    loads = [sum(m.ncells for m in p) for p in parts]
    assert max(loads) - min(loads) <= max(sizes)  # the largest-first greedy bound
