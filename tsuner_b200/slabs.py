"""Row-slab decomposition of one grid over several GPUs (one process per GPU).

The reference runs one grid on one GPU (GPU/main_TSUNER.cu:55).  Here a grid
of npy rows is split into row slabs, one per rank of a torch.distributed
group; each slab is a solver of libtsuner_b200.so (tsu_slab_create) that owns
its rows and stores two ghost rows on every side that has a neighbour.  Per
time step, for each of the two RK stages:

    exchange the ghost rows of the state the stage reads   (NCCL send/recv)
    run the fused stage kernel on the owned rows            (tsu_slab_stage)

and after the second stage the slabs' dt values are reduced to their minimum
(an 8-byte MIN all-reduce).  The ghost rows travel as contiguous messages
([5 planes][2 rows][npx] doubles) packed and unpacked on the GPU by the
library, sent by NCCL into the neighbour's own device buffer (no peer loads,
no TMA of remote memory).  The mask's ghost rows are exchanged once, after
it is set.  Every rank issues the same collective steps in the same order.

A SlabGroup can also hold several slabs in one process (dist=None): their
ghost rows are then copied between them directly, which is how one GPU tests
the decomposition against the undecomposed solver.  The compute backend is
DeviceSlab (the product library); tests substitute a CPU restatement to check
the exchange logic without a GPU.
"""
import ctypes as C

import numpy as np

from . import _ck, _p, lib

UP, DOWN = 0, 1  # message directions: a slab's north rows go up, its south rows go down


def split_rows(npy, nslabs):
    """Global row ranges [(j0, j1)] of nslabs near-equal slabs (each >= 2 rows)."""
    if nslabs < 1 or npy < 2 * nslabs:
        raise ValueError("%d rows cannot be split into %d slabs of at least 2 rows" % (npy, nslabs))
    cuts = [npy * k // nslabs for k in range(nslabs + 1)]
    return [(cuts[k], cuts[k + 1]) for k in range(nslabs)]


def neighbours(k, nslabs, periodic):
    """(south, north) slab indices of slab k, None where the grid ends."""
    south = k - 1 if k > 0 else (nslabs - 1 if periodic else None)
    north = k + 1 if k < nslabs - 1 else (0 if periodic else None)
    return south, north


class DeviceSlab:
    """One row slab on one GPU through the tsu_slab_* C ABI.  Its work is
    issued on the current torch stream of its device, the stream the
    messages use too."""

    def __init__(self, p, sw, j0, j1, device=0):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.p, self.sw, self.j0, self.j1 = p, sw, j0, j1
        self._h = C.c_void_p()
        _ck(lib().tsu_slab_create(C.byref(self._h), C.byref(p), C.byref(sw), j0, j1, device), "tsu_slab_create")
        info = [C.c_int() for _ in range(4)]
        _ck(lib().tsu_slab_info(self._h, *[C.byref(x) for x in info]), "tsu_slab_info")
        self.gs, self.gn = info[2].value, info[3].value
        with torch.cuda.device(self.dev):
            stream = torch.cuda.current_stream(self.dev)
            _ck(lib().tsu_set_stream(self._h, C.c_void_p(stream.cuda_stream)), "tsu_set_stream")
        self._send, self._recv = {}, {}
        for which in (0, 1, 2):
            n = C.c_size_t()
            _ck(lib().tsu_slab_halo_bytes(self._h, which, C.byref(n)), "tsu_slab_halo_bytes")
            dt = torch.uint8 if which == 2 else torch.float64
            count = n.value // (1 if which == 2 else 8)
            for side in (0, 1):
                self._send[which, side] = torch.empty(count, dtype=dt, device=self.dev)
                self._recv[which, side] = torch.empty(count, dtype=dt, device=self.dev)
        self._dt = torch.empty(1, dtype=torch.float64, device=self.dev)

    def close(self):
        if self._h:
            lib().tsu_destroy(self._h)
        self._h = C.c_void_p()

    def set_state(self, V):
        V = np.ascontiguousarray(V, np.float64)
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

    def stage(self, k):
        _ck(lib().tsu_slab_stage(self._h, k), "tsu_slab_stage")

    def pack(self, which, side):
        buf = self._send[which, side]
        _ck(lib().tsu_slab_pack(self._h, which, side, C.c_void_p(buf.data_ptr())), "tsu_slab_pack")
        return buf

    def recv_buffer(self, which, side):
        return self._recv[which, side]

    def unpack(self, which, side):
        buf = self._recv[which, side]
        _ck(lib().tsu_slab_unpack(self._h, which, side, C.c_void_p(buf.data_ptr())), "tsu_slab_unpack")

    def dt_buffer(self):
        _ck(lib().tsu_get_dt_device(self._h, C.c_void_p(self._dt.data_ptr())), "tsu_get_dt_device")
        return self._dt

    def set_dt(self, d):
        _ck(lib().tsu_set_dt_device(self._h, C.c_void_p(d.data_ptr())), "tsu_set_dt_device")

    def sync(self):
        self.torch.cuda.current_stream(self.dev).synchronize()
        _ck(lib().tsu_sync(self._h), "tsu_sync")

    def state(self):
        V = np.empty((5, self.j1 - self.j0, self.p.npx))
        _ck(lib().tsu_get_state(self._h, _p(V)), "tsu_get_state")
        return V

    def extrema(self):
        shp = (self.j1 - self.j0, self.p.npx)
        a, b, c = np.empty(shp), np.empty(shp), np.empty(shp)
        _ck(lib().tsu_get_extrema(self._h, _p(a), _p(b), _p(c)), "tsu_get_extrema")
        return a, b, c

    def time(self):
        t, dt, n = C.c_double(), C.c_double(), C.c_long()
        _ck(lib().tsu_get_time(self._h, C.byref(t), C.byref(dt), C.byref(n)), "tsu_get_time")
        return t.value, dt.value, n.value


class SlabGroup:
    """The slabs of one grid held by this process, stepped together.

    dist: an initialised torch.distributed (one slab per rank: rank k holds
    slab k, messages to other ranks go by send/recv); None: all nslabs slabs
    live in this process.  backend(p, sw, j0, j1, device) makes one slab
    (default DeviceSlab)."""

    def __init__(self, p, sw, nslabs=None, dist=None, device=0, backend=None):
        self.p, self.sw, self.dist = p, sw, dist
        if dist is not None:
            self.nslabs = dist.get_world_size()
            self.local = [dist.get_rank()]
        else:
            self.nslabs = int(nslabs)
            self.local = list(range(self.nslabs))
        self.rows = split_rows(p.npy, self.nslabs)
        self.periodic = (sw.wbc == 2)
        if self.periodic and self.nslabs < 2:
            raise ValueError("a periodic grid needs at least 2 slabs")
        make = backend or DeviceSlab
        self.slabs = {k: make(p, sw, self.rows[k][0], self.rows[k][1], device) for k in self.local}

    def close(self):
        for s in self.slabs.values():
            close = getattr(s, "close", None)
            if close:
                close()

    # -------------------------------------------------------------- set-up
    def load(self, V, mask=None, CC=None, tCC=None):
        """Whole-grid host state (5, npy, npx), mask (npy, npx), series."""
        for k, s in self.slabs.items():
            j0, j1 = self.rows[k]
            s.set_state(V[:, j0:j1])
            s.set_mask(None if mask is None else mask[j0:j1])
            if self.sw.read_files:
                s.set_boundary_series(CC, tCC)
        self.exchange(2)

    def reset(self):
        for s in self.slabs.values():
            s.reset()
        self.reduce_dt()

    # -------------------------------------------------------------- stepping
    def step(self, n=1):
        for _ in range(n):
            for k in range(2):
                self.exchange(k)  # buffer k is what stage k reads
                for s in self.slabs.values():
                    s.stage(k)
            self.reduce_dt()

    def exchange(self, which):
        """Fills every local slab's ghost rows of buffer `which` from its
        neighbours.  Messages are posted in a fixed order (sends: up, then
        down; receives: from below, then from above), so that two messages
        between the same pair of ranks are matched in order."""
        ops, unpack = [], []
        dist = self.dist
        for k in self.local:
            s = self.slabs[k]
            south, north = neighbours(k, self.nslabs, self.periodic)
            for side, nb, tag in ((1, north, UP), (0, south, DOWN)):
                if nb is None:
                    continue
                buf = s.pack(which, side)
                if nb in self.slabs:  # the neighbour is here: a device-local copy
                    self.slabs[nb].recv_buffer(which, 1 - side).copy_(buf)
                    unpack.append((nb, 1 - side))
                else:
                    ops.append(dist.P2POp(dist.isend, buf, nb, tag=4 * which + tag))
        for k in self.local:
            s = self.slabs[k]
            south, north = neighbours(k, self.nslabs, self.periodic)
            for side, nb, tag in ((0, south, UP), (1, north, DOWN)):
                if nb is None or nb in self.slabs:
                    continue
                ops.append(dist.P2POp(dist.irecv, s.recv_buffer(which, side), nb, tag=4 * which + tag))
                unpack.append((k, side))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        for k, side in unpack:
            self.slabs[k].unpack(which, side)

    def reduce_dt(self):
        """The grid's next dt: the minimum of the slabs' (each rounded as the
        whole grid's), given back to every slab."""
        vals = [s.dt_buffer() for s in self.slabs.values()]
        m = vals[0].clone()
        for v in vals[1:]:
            m = m.minimum(v)
        if self.dist is not None:
            self.dist.all_reduce(m, op=self.dist.ReduceOp.MIN)
        for s in self.slabs.values():
            s.set_dt(m)

    def sync(self):
        for s in self.slabs.values():
            s.sync()

    # -------------------------------------------------------------- read-back
    def local_state(self):
        """{slab index: (j0, owned state (5, rows, npx))} of this process."""
        return {k: (self.rows[k][0], s.state()) for k, s in self.slabs.items()}

    def local_extrema(self):
        return {k: (self.rows[k][0],) + tuple(s.extrema()) for k, s in self.slabs.items()}

    def time(self):
        """(t, dt, steps) of the first local slab (every slab holds the same)."""
        return self.slabs[self.local[0]].time()
