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

    def close(self):
        if self.h:
            _lib.tempi().tempi_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


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
