"""CPU: the multi-process plumbing of bench.py (replicas only) with the gloo
backend at world size 2: every rank joins, the barrier completes, and the
reported time is the maximum over ranks."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
mp = torch.multiprocessing


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    r, w, local, dist = bench.dist_setup(world, backend="gloo")
    try:
        bench.barrier(dist, local)
        ms = 10.0 + 5.0 * r  # rank-dependent device time
        out.put((r, w, bench.dist_max(dist, ms, local)))
        bench.barrier(dist, local)
    finally:
        dist.destroy_process_group()


def test_replicas_barrier_and_max_over_ranks():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    os.environ["PYTHONPATH"] = root + os.pathsep + os.environ.get("PYTHONPATH", "")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(0, 2, 15.0), (1, 2, 15.0)]


def test_single_process_is_not_distributed():
    import bench
    saved = os.environ.pop("RANK", None)
    try:
        assert bench.dist_setup(1) == (0, 1, int(os.environ.get("LOCAL_RANK", 0)), None)
        assert bench.dist_max(None, 3.5, 0) == 3.5
    finally:
        if saved is not None:
            os.environ["RANK"] = saved
