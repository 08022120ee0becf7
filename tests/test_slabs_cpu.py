"""CPU: the row-slab decomposition of one grid (tsuner_b200/slabs.py), its
halo exchange and its dt reduction, with the oracle as the compute backend
(oracle.OracleSlab), against a single-grid oracle run of the same inputs.

The decomposition must not change a single value: after the run every owned
cell, the running extrema, the simulated time and the next dt equal the
undecomposed run's.  Covered: walls with the CC boundary series and a
harbour mask (the series segments of the west/east boundaries lie in every
slab), free boundaries, a periodic grid (the seam between the last and the
first slab), uneven slab heights, slabs of 2 rows, and the float-rounded dt
of grids above 4096 cells.  Once with all slabs in one process (direct ghost
row copies) and once as a gloo group of two processes (send/recv and a MIN
all-reduce), the path the GPUs take with NCCL."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
mp = torch.multiprocessing

import oracle  # noqa: E402
from tsuner_b200 import slabs as S  # noqa: E402
from tsuner_b200 import workloads as W  # noqa: E402
from tsuner_b200.abi import make_switches  # noqa: E402


def case(name):
    if name == "nwave_walls":
        w = W.nwave_shelf(40, 29, 40.0, slr=0.5, amp=2.0, period=200.0, t_series=150.0)
        return w, w.sw
    if name == "free":
        w = W.hump(36, 26, 10.0, sigma=60.0)
        return w, make_switches(order=2, wbc=0, read_files=0)
    if name == "periodic_series":
        w = W.nwave_shelf(32, 24, 40.0, slr=0.5, amp=1.0, period=200.0, t_series=120.0)
        return w, make_switches(order=2, wbc=2, read_files=1)
    if name == "periodic":
        w = W.hump(30, 22, 10.0, sigma=50.0)
        return w, make_switches(order=2, wbc=2, read_files=0)
    raise KeyError(name)


def whole_grid(w, sw, steps):
    r = oracle.OracleRun(w.p, sw, w.V, w.mask, w.CC if sw.read_files else None, w.tCC if sw.read_files else None)
    r.run(steps)
    shp = (w.p.npy, w.p.npx)
    return r.V, (r.hmax.reshape(shp), r.bmin.reshape(shp), r.eta_max.reshape(shp)), r.t.value, r.dt.value


def assemble(w, parts):
    V = np.full((5, w.p.npy, w.p.npx), np.nan)
    for j0, Vs in parts.values():
        V[:, j0:j0 + Vs.shape[1]] = Vs
    return V


@pytest.mark.parametrize("name,nslabs", [("nwave_walls", 2), ("nwave_walls", 3), ("free", 4), ("periodic", 2),
                                         ("periodic", 3), ("periodic_series", 2)])
def test_slabs_in_one_process_equal_the_whole_grid(name, nslabs):
    w, sw = case(name)
    g = S.SlabGroup(w.p, sw, nslabs=nslabs, backend=oracle.OracleSlab)
    g.load(w.V, w.mask, w.CC, w.tCC)
    g.reset()
    g.step(25)
    V = assemble(w, g.local_state())
    ext = {k: v for k, v in g.local_extrema().items()}
    t, dt, n = g.time()
    Vr, er, tr, dtr = whole_grid(w, sw, 25)
    assert n == 25
    assert np.array_equal(V, Vr)
    assert t == tr and dt == dtr
    for k, (j0, hmax, bmin, eta) in ext.items():
        rows = slice(j0, j0 + hmax.shape[0])
        assert np.array_equal(hmax, er[0][rows]) and np.array_equal(bmin, er[1][rows])
        assert np.array_equal(eta, er[2][rows])


def test_two_row_slabs_and_uneven_split():
    assert S.split_rows(29, 3) == [(0, 9), (9, 19), (19, 29)]
    assert S.neighbours(0, 3, False) == (None, 1) and S.neighbours(2, 3, True) == (1, 0)
    with pytest.raises(ValueError):
        S.split_rows(5, 3)
    w = W.hump(20, 8, 10.0, sigma=30.0)
    g = S.SlabGroup(w.p, w.sw, nslabs=4, backend=oracle.OracleSlab)  # four slabs of 2 rows
    g.load(w.V, w.mask)
    g.reset()
    g.step(15)
    Vr, _, tr, _ = whole_grid(w, w.sw, 15)
    assert np.array_equal(assemble(w, g.local_state()), Vr)
    assert g.time()[0] == tr


def test_dt_rounding_follows_the_whole_grid():
    """72 x 64 = 4608 cells: the reference rounds the dt minimum to float; each
    slab alone has fewer than 4096 cells but must round as the grid does."""
    w = W.hump(72, 64, 10.0, sigma=120.0)
    g = S.SlabGroup(w.p, w.sw, nslabs=2, backend=oracle.OracleSlab)
    g.load(w.V, w.mask)
    g.reset()
    dt0 = g.time()[1]
    assert dt0 == float(np.float32(dt0))
    assert dt0 == oracle.initial_dt(w.p, w.sw, w.V)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, name, steps, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        w, sw = case(name)
        g = S.SlabGroup(w.p, sw, dist=dist, backend=oracle.OracleSlab)
        g.load(w.V, w.mask, w.CC, w.tCC)
        g.reset()
        g.step(steps)
        dist.barrier()
        out.put((rank, g.local_state(), g.time()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", ["nwave_walls", "periodic_series"])
def test_gloo_two_ranks_equal_the_whole_grid(name):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    os.environ["PYTHONPATH"] = root + os.pathsep + os.environ.get("PYTHONPATH", "")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, name, 20, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=180) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    w, sw = case(name)
    parts = {}
    times = set()
    for rank, st, t in res:
        parts.update(st)
        times.add(t)
    assert len(times) == 1  # every rank holds the same t, dt and step count
    Vr, _, tr, dtr = whole_grid(w, sw, 20)
    assert np.array_equal(assemble(w, parts), Vr)
    t, dt, n = times.pop()
    assert (t, dt, n) == (tr, dtr, 20)
