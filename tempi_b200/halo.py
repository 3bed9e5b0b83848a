"""Halo regions of 3-D grids as MPI subarray types, and batched packing.

A grid has an interior of nx x ny x nz cells and a ghost layer of `radius`
cells on every side; it is stored C-order with x fastest, so the allocation
is (nz+2r, ny+2r, nx+2r) elements.  Each of the 26 neighbour directions
(6 faces, 12 edges, 8 corners) has a send region (interior cells the
neighbour needs) and a receive region (ghost cells filled from that
neighbour), both committed MPI_Type_create_subarray types -- the layout of the
reference's halo benchmark (bin/bench_halo_exchange.cpp).

``HaloBatch`` packs every region of one or several grids with one kernel
launch through tempi_batch_* (and can replay it from a CUDA graph);
``pack_plain`` does the same with one MPI_Pack call per region, the
reference's per-call path.

A grid whose neighbours in every direction are the grid itself (one rank,
periodic boundaries, as the reference's halo benchmark runs at world size 1)
exchanges its halo by copying each send region into the ghost region on the
opposite side.  ``HaloExchange`` does that with the fused copy kernel
(tempi_batch_create_copy: no packed buffer, one launch); ``exchange_alltoallw``
does it through the interposed MPI_Neighbor_alltoallw over a graph
communicator with 26 self-edges; ``exchange_plain`` is the reference's
sequence (26 MPI_Pack, MPI_Neighbor_alltoallv of the packed bytes, 26
MPI_Unpack; bin/bench_halo_exchange.cpp:560-625).
"""
from __future__ import annotations

import ctypes
import itertools

from . import _lib, mpi


def directions():
    """The 26 (dx, dy, dz) neighbour directions, in a fixed order."""
    return [d for d in itertools.product((-1, 0, 1), repeat=3) if d != (0, 0, 0)]


def _axis(n, r, d, ghost):
    if d == 0:
        return r, n
    if ghost:
        return (0, r) if d < 0 else (n + r, r)
    return (r, r) if d < 0 else (n, r)


class Grid:
    """One grid and its 52 committed region types (26 send, 26 receive)."""

    def __init__(self, interior, radius, elem=mpi.DOUBLE, elem_bytes=8):
        self.n = tuple(int(x) for x in interior)  # (nx, ny, nz)
        self.r = int(radius)
        self.elem = elem
        self.elem_bytes = elem_bytes
        nx, ny, nz = self.n
        r = self.r
        self.alloc = (nx + 2 * r, ny + 2 * r, nz + 2 * r)
        self.nbytes = self.alloc[0] * self.alloc[1] * self.alloc[2] * elem_bytes
        self.send, self.recv, self.region_shape = {}, {}, {}
        sizes = [self.alloc[2], self.alloc[1], self.alloc[0]]
        for d in directions():
            for ghost, table in ((False, self.send), (True, self.recv)):
                ax = [_axis(self.n[i], r, d[i], ghost) for i in range(3)]
                starts = [ax[2][0], ax[1][0], ax[0][0]]
                subs = [ax[2][1], ax[1][1], ax[0][1]]
                t = mpi.Type_create_subarray(sizes, subs, starts, mpi.ORDER_C, elem)
                assert mpi.Type_commit(t) == 0
                table[d] = t
                self.region_shape[(d, ghost)] = (subs, starts)
        self.region_bytes = {
            d: mpi.Type_size(self.send[d]) for d in directions()
        }
        self.packed_bytes = sum(self.region_bytes.values())

    def offsets(self):
        """Packed offset of each direction's send region."""
        out, pos = {}, 0
        for d in directions():
            out[d] = pos
            pos += self.region_bytes[d]
        return out


def mixed_shapes(seed=8, count=8):
    """(interior, radius) of the mixed halo batch: `count` grids whose
    interior dimensions are each drawn log-uniform from [32, 512] and whose
    radius is drawn from 1..3, all from one seed."""
    import numpy as np

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        interior = [int(round(np.exp(rng.uniform(np.log(32), np.log(512))))) for _ in range(3)]
        out.append((interior, int(rng.integers(1, 4))))
    return out


def regions(grids, grid_ptrs, packed_ptrs, unpack=False):
    """tempi_region entries for every region of every grid.  For unpack the
    bytes packed for direction d land in the ghost region of direction -d
    (what a periodic neighbour exchange delivers)."""
    out = []
    for g, gp, pp in zip(grids, grid_ptrs, packed_ptrs):
        offs = g.offsets()
        for d in directions():
            t = g.recv[tuple(-x for x in d)] if unpack else g.send[d]
            err, desc = mpi.describe(t)
            _lib.check(err, "tempi_describe")
            r = _lib.Region()
            r.origin = gp
            r.packed = pp + offs[d]
            r.desc = desc
            r.incount = 1
            out.append(r)
    return out


class HaloBatch:
    """One batched pack (or unpack) of all regions of `grids`."""

    def __init__(self, grids, grid_ptrs, packed_ptrs, unpack=False):
        regs = regions(grids, grid_ptrs, packed_ptrs, unpack)
        arr = (_lib.Region * len(regs))(*regs)
        h = ctypes.c_void_p()
        _lib.check(_lib.tempi().tempi_batch_create(arr, len(regs), int(unpack),
                                                   ctypes.byref(h)), "tempi_batch_create")
        self.h = h
        self.nregions = len(regs)

    def launch(self, stream=None):
        _lib.check(_lib.tempi().tempi_batch_launch(self.h, stream), "tempi_batch_launch")

    def capture(self, stream):
        _lib.check(_lib.tempi().tempi_batch_capture(self.h, stream), "tempi_batch_capture")

    def replay(self, stream):
        _lib.check(_lib.tempi().tempi_batch_replay(self.h, stream), "tempi_batch_replay")

    def tune(self, stream=None, reps=5):
        """Time the launch shapes and per-class chunk passes (tempi_batch_tune)
        and keep the fastest; a captured graph must be captured again."""
        _lib.check(_lib.tempi().tempi_batch_tune(self.h, stream, reps), "tempi_batch_tune")

    def config(self):
        """(threads per block, blocks per SM, {region class: passes})."""
        th, cps = ctypes.c_int32(), ctypes.c_int32()
        cls, ps = (ctypes.c_int32 * 40)(), (ctypes.c_int32 * 40)()
        n = _lib.tempi().tempi_batch_config(self.h, ctypes.byref(th), ctypes.byref(cps), cls,
                                            ps, 40)
        if n < 0:
            raise RuntimeError(_lib.last_error())
        return th.value, cps.value, {cls[i]: ps[i] for i in range(n)}

    def close(self):
        if self.h:
            _lib.tempi().tempi_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def copy_regions(grids, grid_ptrs):
    """tempi_copy_region entries for a periodic self-exchange of every grid:
    the send region of direction d goes to the ghost region of -d."""
    out = []
    for g, gp in zip(grids, grid_ptrs):
        for d in directions():
            err, sd = mpi.describe(g.send[d])
            _lib.check(err, "tempi_describe")
            err, rd = mpi.describe(g.recv[tuple(-x for x in d)])
            _lib.check(err, "tempi_describe")
            c = _lib.CopyRegion()
            c.src_origin = gp
            c.dst_origin = gp
            c.src_desc = sd
            c.dst_desc = rd
            c.src_count = 1
            c.dst_count = 1
            out.append(c)
    return out


class HaloExchange(HaloBatch):
    """The whole periodic self-exchange of `grids` in one fused launch; the
    handle launches, captures, replays and closes like a HaloBatch."""

    def __init__(self, grids, grid_ptrs):
        regs = copy_regions(grids, grid_ptrs)
        arr = (_lib.CopyRegion * len(regs))(*regs)
        h = ctypes.c_void_p()
        _lib.check(_lib.tempi().tempi_batch_create_copy(arr, len(regs), ctypes.byref(h)),
                   "tempi_batch_create_copy")
        self.h = h
        self.nregions = len(regs)


class SelfGraph:
    """A graph communicator with 26 self-edges (one per direction) and the
    per-edge arguments of MPI_Neighbor_alltoallv / MPI_Neighbor_alltoallw for
    one grid."""

    def __init__(self, grid: Grid):
        n = len(directions())
        err, self.comm = mpi.Dist_graph_create_adjacent([0] * n, [0] * n)
        _lib.check(err, "MPI_Dist_graph_create_adjacent")
        self.grid = grid
        offs = grid.offsets()
        self.counts = [grid.region_bytes[d] for d in directions()]
        self.displs = [offs[d] for d in directions()]
        self.sendtypes = [grid.send[d] for d in directions()]
        self.recvtypes = [grid.recv[tuple(-x for x in d)] for d in directions()]

    def close(self):
        if self.comm:
            mpi.Comm_free(self.comm)
            self.comm = 0


def exchange_alltoallw(g: SelfGraph, grid_ptr: int) -> None:
    n = len(g.sendtypes)
    err = mpi.Neighbor_alltoallw(grid_ptr, [1] * n, [0] * n, g.sendtypes, grid_ptr,
                                 [1] * n, [0] * n, g.recvtypes, g.comm)
    if err:
        raise RuntimeError(f"MPI_Neighbor_alltoallw failed: {err} {_lib.last_error()}")


def exchange_plain(g: SelfGraph, grid_ptr: int, sendbuf: int, recvbuf: int) -> None:
    """The reference's sequence: pack every region, exchange the packed bytes
    with MPI_Neighbor_alltoallv, unpack every region."""
    pack_plain(g.grid, grid_ptr, sendbuf)
    err = mpi.Neighbor_alltoallv(sendbuf, g.counts, g.displs, mpi.BYTE, recvbuf, g.counts,
                                 g.displs, mpi.BYTE, g.comm)
    if err:
        raise RuntimeError(f"MPI_Neighbor_alltoallv failed: {err}")
    unpack_plain(g.grid, recvbuf, grid_ptr)


def pack_plain(grid: Grid, grid_ptr: int, packed_ptr: int) -> int:
    """26 MPI_Pack calls, one per region, the reference's per-call path."""
    pos = 0
    for d in directions():
        err, pos = mpi.Pack(grid_ptr, 1, grid.send[d], packed_ptr, grid.packed_bytes, pos)
        if err:
            raise RuntimeError(f"MPI_Pack failed: {err} {_lib.last_error()}")
    return pos


def unpack_plain(grid: Grid, packed_ptr: int, grid_ptr: int) -> int:
    offs = grid.offsets()
    for d in directions():
        t = grid.recv[tuple(-x for x in d)]
        err, _ = mpi.Unpack(packed_ptr, grid.packed_bytes, grid_ptr, 1, t, offs[d])
        if err:
            raise RuntimeError(f"MPI_Unpack failed: {err} {_lib.last_error()}")
    return grid.packed_bytes
