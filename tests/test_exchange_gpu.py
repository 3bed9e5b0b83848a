"""The fused exchange (tempi_batch_create_copy: each region copied from one
strided layout straight into another in one launch) and the interposed
MPI_Neighbor_alltoallw built on it, against the oracle's pack followed by
its unpack.  Gap bytes of the destination keep their 0xAA fill."""
import ctypes

import numpy as np
import pytest

from oracle import types as T
from tempi_b200 import _lib, halo, mpi

from . import helpers as H
from .test_batch_gpu import oracle_grid_types
from .test_canon import desc_pack

pytestmark = pytest.mark.gpu


def desc_unpack(d, packed, buf, incount):
    shape = [incount] + [d.counts[k] for k in reversed(range(d.ndims))] + [d.block]
    strides = [d.extent] + [d.strides[k] for k in reversed(range(d.ndims))] + [1]
    v = np.lib.stride_tricks.as_strided(buf[d.start:], shape=shape, strides=strides,
                                        writeable=True)
    v[...] = packed.reshape(v.shape)


def test_copy_between_different_layouts(cuda, mpi_init):
    """Source and destination layouts differ in row length, stride, count and
    alignment (so the two geometries decompose the same word index
    differently), including odd starts that force 1-byte words."""
    import torch

    cases = [  # (src desc, src count, dst desc, dst count)
        (_lib.Desc.make(12, 5000, 24, [100], [40]), 2,
         _lib.Desc.make(4, 9000, 16, [300], [24]), 1),
        (_lib.Desc.make(3, 7000, 60, [7, 9], [64, 700]), 1,
         _lib.Desc.make(1, 8000, 35, [108], [41]), 1),
        (_lib.Desc.make(0, 1 << 16, 4096, [8], [8192]), 1,
         _lib.Desc.make(16, 40000, 1024, [32], [1040]), 1),
        (_lib.Desc.make(8, 2048, 8, [16], [16]), 3,
         _lib.Desc.make(0, 6000, 12, [32], [20]), 1),
    ]
    def span(d, n):
        return d.start + (n - 1) * d.extent + sum(
            (d.counts[k] - 1) * d.strides[k] for k in range(d.ndims)) + d.block

    for sd, sc, dd, dc in cases:
        assert sd.size * sc == dd.size * dc
        assert span(sd, sc) <= sd.extent * sc and span(dd, dc) <= dd.extent * dc
        src_np = H.splitmix_bytes(sd.extent * sc + 64, sd.block)
        dst_np = np.full(dd.extent * dc + 64, 0xAA, np.uint8)
        src = torch.from_numpy(src_np).cuda()
        dst = torch.from_numpy(dst_np.copy()).cuda()
        r = _lib.CopyRegion()
        r.src_origin, r.dst_origin = src.data_ptr(), dst.data_ptr()
        r.src_desc, r.dst_desc, r.src_count, r.dst_count = sd, dd, sc, dc
        arr = (_lib.CopyRegion * 1)(r)
        h = ctypes.c_void_p()
        _lib.check(_lib.tempi().tempi_batch_create_copy(arr, 1, ctypes.byref(h)))
        _lib.check(_lib.tempi().tempi_batch_launch(h, None))
        torch.cuda.synchronize()
        _lib.tempi().tempi_batch_destroy(h)
        want = dst_np.copy()
        desc_unpack(dd, desc_pack(sd, src_np, sc), want, dc)
        assert dst.cpu().numpy().tobytes() == want.tobytes(), (sd.block, dd.block)


def test_copy_rejects_size_mismatch(cuda, mpi_init):
    r = _lib.CopyRegion()
    r.src_desc = _lib.Desc.make(0, 100, 10, [5], [20])
    r.dst_desc = _lib.Desc.make(0, 100, 10, [4], [20])
    r.src_count = r.dst_count = 1
    h = ctypes.c_void_p()
    assert _lib.tempi().tempi_batch_create_copy((_lib.CopyRegion * 1)(r), 1, ctypes.byref(h)) != 0


def oracle_exchange(g, data):
    ts = oracle_grid_types(g, False)
    tr = oracle_grid_types(g, True)
    out = data.copy()
    for d in halo.directions():
        T.unpack(tr[tuple(-x for x in d)], T.pack(ts[d], data, 1), out, 1)
    return out


@pytest.mark.parametrize("interior,radius", [((20, 17, 9), 2), ((33, 8, 12), 1), ((16, 16, 16), 3)])
def test_periodic_self_exchange_fused_alltoallw_and_plain(cuda, mpi_init, interior, radius):
    import torch

    g = halo.Grid(interior, radius)
    data_np = H.splitmix_bytes(g.nbytes, radius + 40)
    want = oracle_exchange(g, data_np)
    # fused kernel, launched and replayed from a graph
    a = torch.from_numpy(data_np).cuda()
    x = halo.HaloExchange([g], [a.data_ptr()])
    assert x.nregions == 26
    x.launch()
    torch.cuda.synchronize()
    assert a.cpu().numpy().tobytes() == want.tobytes()
    s = torch.cuda.Stream()
    a.copy_(torch.from_numpy(data_np))
    torch.cuda.synchronize()
    x.capture(s.cuda_stream)
    x.replay(s.cuda_stream)
    s.synchronize()
    assert a.cpu().numpy().tobytes() == want.tobytes()
    x.close()
    # the interposed MPI_Neighbor_alltoallw: all 26 edges are self-edges
    sg = halo.SelfGraph(g)
    b = torch.from_numpy(data_np).cuda()
    torch.cuda.synchronize()
    n0 = _lib.counter("neighbor_fused")
    halo.exchange_alltoallw(sg, b.data_ptr())
    assert _lib.counter("neighbor_fused") == n0 + 1
    assert b.cpu().numpy().tobytes() == want.tobytes()
    # the same call again (its region table is already on the device) on
    # fresh data
    data2 = H.splitmix_bytes(g.nbytes, radius + 41)
    b.copy_(torch.from_numpy(data2))
    torch.cuda.synchronize()
    halo.exchange_alltoallw(sg, b.data_ptr())
    assert b.cpu().numpy().tobytes() == oracle_exchange(g, data2).tobytes()
    # the reference's sequence through the interposer and the library
    c = torch.from_numpy(data_np).cuda()
    sendbuf = torch.zeros(g.packed_bytes, dtype=torch.uint8, device="cuda")
    recvbuf = torch.zeros_like(sendbuf)
    torch.cuda.synchronize()
    halo.exchange_plain(sg, c.data_ptr(), sendbuf.data_ptr(), recvbuf.data_ptr())
    torch.cuda.synchronize()
    assert c.cpu().numpy().tobytes() == want.tobytes()
    sg.close()


def test_alltoallw_mixed_edges_use_isir(cuda, mpi_init):
    """An undescribable type (a struct of two different blocks) on one edge
    keeps the call off the fused kernel: the reference's Isend/Irecv sequence
    runs, still bit-exact."""
    import torch

    err, comm = mpi.Dist_graph_create_adjacent([0, 0], [0, 0])
    assert err == 0
    vec = H.vector(64, 3, 7, H.named("BYTE")).commit()
    st = H.struct([2, 5], [0, 16], [H.named("BYTE"), H.named("BYTE")]).commit()
    buf_np = H.splitmix_bytes(4096, 9)
    buf = torch.from_numpy(buf_np).cuda()
    out = torch.full((4096,), 0xAA, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    n0 = _lib.counter("neighbor_isir")
    assert mpi.Neighbor_alltoallw(buf.data_ptr(), [1, 1], [0, 1000], [vec.h, st.h],
                                  out.data_ptr(), [1, 1], [100, 3000], [vec.h, st.h],
                                  comm) == 0
    assert _lib.counter("neighbor_isir") == n0 + 1
    want = np.full(4096, 0xAA, np.uint8)
    T.unpack(vec.o, T.pack(vec.o, buf_np, 1), want, 1, origin=100)
    T.unpack(st.o, T.pack(st.o, buf_np, 1, origin=1000), want, 1, origin=3000)
    assert out.cpu().numpy().tobytes() == want.tobytes()
    mpi.Comm_free(comm)


def _rand_desc(rng, max_bytes):
    """A seeded random non-overlapping descriptor of at most `max_bytes`
    described bytes: 0-3 strided dimensions at any alignment."""
    while True:
        nd = int(rng.integers(0, 4))
        block = int(rng.integers(1, 300 if nd else 5000))
        counts, strides, span = [], [], block
        for _ in range(nd):
            c = int(rng.integers(1, 20))
            st = span + int(rng.integers(0, 24))
            counts.append(c)
            strides.append(st)
            span = st * (c - 1) + span
        d = _lib.Desc.make(int(rng.integers(0, 20)), span + int(rng.integers(0, 20)),
                           block, counts, strides)
        if 0 < d.size <= max_bytes:
            return d


def test_copy_batch_random_pairs(cuda, mpi_init):
    """One fused copy of 40 seeded random (source layout, destination layout)
    pairs of equal byte counts -- the destination a row layout of a different
    row length and alignment -- into one destination buffer: every pair's
    bytes arrive in type-map order, and no other byte changes."""
    import torch

    rng = np.random.default_rng(31337)
    srcs, dsts, pairs = [], [], []
    sbase = dbase = 0
    for i in range(40):
        sd = _rand_desc(rng, 200000)
        sc = int(rng.integers(1, 4))
        total = sd.size * sc
        divisors = [b for b in range(1, min(total, 4096) + 1) if total % b == 0]
        bl = int(rng.choice(divisors))
        cnt = total // bl
        st = bl + int(rng.integers(0, 40))
        dd = _lib.Desc.make(int(rng.integers(0, 16)), st * cnt + 16, bl, [cnt], [st])
        srcs.append((sbase, sd, sc))
        dsts.append((dbase, dd))
        sbase += sd.extent * sc + 64
        dbase += dd.extent + 64
    src_np = H.splitmix_bytes(sbase, 4242)
    dst_np = np.full(dbase, 0xAA, np.uint8)
    src = torch.from_numpy(src_np).cuda()
    dst = torch.from_numpy(dst_np.copy()).cuda()
    arr = (_lib.CopyRegion * 40)()
    for k, ((sb, sd, sc), (db, dd)) in enumerate(zip(srcs, dsts)):
        r = arr[k]
        r.src_origin, r.dst_origin = src.data_ptr() + sb, dst.data_ptr() + db
        r.src_desc, r.dst_desc, r.src_count, r.dst_count = sd, dd, sc, 1
    h = ctypes.c_void_p()
    _lib.check(_lib.tempi().tempi_batch_create_copy(arr, 40, ctypes.byref(h)))
    _lib.check(_lib.tempi().tempi_batch_launch(h, None))
    torch.cuda.synchronize()
    _lib.tempi().tempi_batch_destroy(h)
    want = dst_np.copy()
    for (sb, sd, sc), (db, dd) in zip(srcs, dsts):
        seg = want[db: db + dd.extent + 64]
        desc_unpack(dd, desc_pack(sd, src_np[sb: sb + sd.extent * sc + 64], sc), seg, 1)
    assert dst.cpu().numpy().tobytes() == want.tobytes()
