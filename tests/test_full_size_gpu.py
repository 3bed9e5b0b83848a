"""Parity at the benchmark configurations' full sizes, against the oracle's
multi-threaded C type-map walker (oracle/typemap.c):

* the 26-region halo of a 256^3 grid of doubles with radius 2 (140.6 MB
  allocation, 6,390,272 B packed): pack by 26 plain MPI_Pack calls, by one
  batched launch and by a CUDA-graph replay with new data; unpack into the
  ghost cells the same three ways;
* the benchmark's own mixed batch of 8 grids (interiors log-uniform in
  32..512 per dimension, radius 1..3, the benchmark's seed), packed and
  unpacked in one launch and by graph replay;
* every point of the benchmark's strided sweep (its exact subarrays and
  starts) through the interposed MPI_Pack / MPI_Unpack at incount 1, 4 and
  16: up to 1 GiB of typed data per call, where 64-bit offsets matter.

Every comparison is of whole buffers: packed bytes, and unpack destinations
prefilled with 0xAA (or holding the grid's interior) outside the described
bytes."""
import os

import numpy as np
import pytest

from oracle import types as T
from oracle import walker as W
from tempi_b200 import halo, mpi

from . import helpers as H

pytestmark = pytest.mark.gpu

NT = max(1, min(32, len(os.sched_getaffinity(0))))


def _walkers(g, ghost):
    sizes = [g.alloc[2], g.alloc[1], g.alloc[0]]
    out = {}
    for d in halo.directions():
        subs, starts = g.region_shape[(d, ghost)]
        out[d] = W.Walker(T.subarray(sizes, subs, starts, T.ORDER_C, T.named(g.elem_bytes)))
    return out


def oracle_pack(g, data_np):
    ws = _walkers(g, False)
    return np.concatenate([ws[d].pack(data_np, 1, nthreads=NT) for d in halo.directions()])


def oracle_unpack(g, packed_np, data_np):
    """The grid after the bytes packed for direction d land in the ghost
    region of -d (a periodic exchange with itself)."""
    ws = _walkers(g, True)
    offs = g.offsets()
    out = data_np.copy()
    for d in halo.directions():
        w = ws[tuple(-x for x in d)]
        w.unpack(np.ascontiguousarray(packed_np[offs[d]: offs[d] + g.region_bytes[d]]), out, 1,
                 nthreads=NT)
    return out


def _host(t):
    return t.cpu().numpy()


def test_halo_256cube_r2_full_size(cuda, mpi_init):
    import torch

    g = halo.Grid((256, 256, 256), 2)
    assert g.nbytes == 260 ** 3 * 8 and g.packed_bytes == 6390272
    data_np = H.splitmix_bytes(g.nbytes, 2562)
    want = oracle_pack(g, data_np)
    data = torch.from_numpy(data_np).cuda()

    # pack: 26 plain calls, one batched launch, a graph replay with new data
    p_plain = torch.zeros(g.packed_bytes, dtype=torch.uint8, device="cuda")
    assert halo.pack_plain(g, data.data_ptr(), p_plain.data_ptr()) == g.packed_bytes
    assert _host(p_plain).tobytes() == want.tobytes()
    p_batch = torch.full_like(p_plain, 0x5A)
    b = halo.HaloBatch([g], [data.data_ptr()], [p_batch.data_ptr()])
    b.launch()
    torch.cuda.synchronize()
    assert _host(p_batch).tobytes() == want.tobytes()
    s = torch.cuda.Stream()
    b.capture(s.cuda_stream)
    data2_np = H.splitmix_bytes(g.nbytes, 2563)
    data.copy_(torch.from_numpy(data2_np))
    torch.cuda.synchronize()
    b.replay(s.cuda_stream)
    s.synchronize()
    want2 = oracle_pack(g, data2_np)
    assert _host(p_batch).tobytes() == want2.tobytes()
    b.close()

    # unpack into the ghost cells: the grid holds data2 everywhere, the
    # packed bytes are `want` (from the first data)
    exp = oracle_unpack(g, want, data2_np)
    packed = torch.from_numpy(want).cuda()
    grids = [torch.from_numpy(data2_np).cuda() for _ in range(3)]
    halo.unpack_plain(g, packed.data_ptr(), grids[0].data_ptr())
    ub = halo.HaloBatch([g], [grids[1].data_ptr()], [packed.data_ptr()], unpack=True)
    ub.launch()
    ug = halo.HaloBatch([g], [grids[2].data_ptr()], [packed.data_ptr()], unpack=True)
    ug.capture(s.cuda_stream)
    ug.replay(s.cuda_stream)
    s.synchronize()
    torch.cuda.synchronize()
    for k, gg in enumerate(grids):
        assert _host(gg).tobytes() == exp.tobytes(), ("plain", "batched", "graph")[k]
    ub.close()
    ug.close()


def test_mixed_8_grids_benchmark_seed(cuda, mpi_init):
    """The benchmark's mixed batch: 8 grids, 208 regions, one launch."""
    import torch

    shapes = halo.mixed_shapes()
    grids = [halo.Grid(interior, r) for interior, r in shapes]
    nps = [H.splitmix_bytes(g.nbytes, 800 + i) for i, g in enumerate(grids)]
    datas = [torch.from_numpy(x).cuda() for x in nps]
    packs = [torch.full((g.packed_bytes,), 0x5A, dtype=torch.uint8, device="cuda") for g in grids]
    b = halo.HaloBatch(grids, [d.data_ptr() for d in datas], [p.data_ptr() for p in packs])
    assert b.nregions == 208
    s = torch.cuda.Stream()
    b.capture(s.cuda_stream)
    b.replay(s.cuda_stream)
    s.synchronize()
    wants = [oracle_pack(g, x) for g, x in zip(grids, nps)]
    for i, (p, w) in enumerate(zip(packs, wants)):
        assert _host(p).tobytes() == w.tobytes(), i
    b.close()
    # unpack every grid's packed bytes into its ghost cells in one launch
    pk = [torch.from_numpy(w).cuda() for w in wants]
    tgt = [torch.from_numpy(x).cuda() for x in nps]
    ub = halo.HaloBatch(grids, [t.data_ptr() for t in tgt], [p.data_ptr() for p in pk], unpack=True)
    ub.launch()
    torch.cuda.synchronize()
    for i, (g, w, x, t) in enumerate(zip(grids, wants, nps, tgt)):
        assert _host(t).tobytes() == oracle_unpack(g, w, x).tobytes(), i
    ub.close()


def _sweep_points():
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    from bench import sweep_points

    return sweep_points()


@pytest.mark.parametrize("ndim", [2, 3])
def test_benchmark_sweep_every_incount(cuda, mpi_init, ndim):
    """The benchmark's exact sweep points through MPI_Pack / MPI_Unpack on
    device buffers at incount 1, 4 and 16."""
    import torch

    pts = [p for p in _sweep_points() if len(p[1]) == ndim]
    extent = 4 * int(np.prod(pts[0][1]))
    src_np = H.splitmix_bytes(16 * extent, 31 + ndim)
    src = torch.from_numpy(src_np).cuda()
    packed = torch.empty(16 * extent, dtype=torch.uint8, device="cuda")
    dst = torch.empty_like(src)
    for label, sizes, subs, starts, _ in pts:
        t = mpi.Type_create_subarray(sizes, subs, starts, mpi.ORDER_C, mpi.FLOAT)
        assert mpi.Type_commit(t) == 0
        o = T.subarray(sizes, subs, starts, T.ORDER_C, T.FLOAT)
        w = W.Walker(o)
        for n in (1, 4, 16):
            size = o.size * n
            err, pos = mpi.Pack(src.data_ptr(), n, t, packed.data_ptr(), packed.numel(), 0)
            assert err == 0 and pos == size, (label, n, err)
            want = np.empty(size, np.uint8)
            w.pack_into(src_np, n, want, nthreads=NT)
            assert _host(packed[:size]).tobytes() == want.tobytes(), (label, n)
            dst.fill_(0xAA)
            err, _ = mpi.Unpack(packed.data_ptr(), packed.numel(), dst.data_ptr(), n, t, 0)
            assert err == 0, (label, n, err)
            exp = np.full(n * extent, 0xAA, np.uint8)
            w.unpack(want, exp, n, nthreads=NT)
            assert _host(dst[: n * extent]).tobytes() == exp.tobytes(), (label, n)
        mpi.Type_free(t)
