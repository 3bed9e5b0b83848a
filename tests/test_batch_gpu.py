"""Batched halo pack/unpack (the halo workload at test sizes): one launch,
or one CUDA-graph replay, must write exactly what 26 per-region MPI_Pack
calls write, and the unpack must fill exactly the ghost cells."""
import numpy as np
import pytest

from oracle import types as T
from tempi_b200 import _lib, halo, mpi

from . import helpers as H

pytestmark = pytest.mark.gpu


def oracle_grid_types(g: halo.Grid, ghost: bool):
    out = {}
    sizes = [g.alloc[2], g.alloc[1], g.alloc[0]]
    for d in halo.directions():
        subs, starts = g.region_shape[(d, ghost)]
        out[d] = T.subarray(sizes, subs, starts, T.ORDER_C, T.named(g.elem_bytes))
    return out


def oracle_pack(g, data):
    ts = oracle_grid_types(g, False)
    return np.concatenate([T.pack(ts[d], data, 1) for d in halo.directions()])


def oracle_unpack(g, packed, data):
    ts = oracle_grid_types(g, True)
    offs = g.offsets()
    out = data.copy()
    for d in halo.directions():
        t = ts[tuple(-x for x in d)]
        T.unpack(t, packed[offs[d]: offs[d] + t.size], out, 1)
    return out


def test_halo_26_regions_sizes(mpi_init):
    g = halo.Grid((256, 256, 256), 2)
    # 6 faces 256*256*2, 12 edges 256*2*2, 8 corners 2*2*2 doubles
    assert g.packed_bytes == 8 * (6 * 256 * 256 * 2 + 12 * 256 * 4 + 8 * 8) == 6390272


@pytest.mark.parametrize("interior,radius", [((20, 17, 9), 2), ((33, 8, 12), 1), ((16, 16, 16), 3)])
def test_batch_matches_plain_and_oracle(cuda, mpi_init, interior, radius):
    import torch

    g = halo.Grid(interior, radius)
    data_np = H.splitmix_bytes(g.nbytes, radius)
    data = torch.from_numpy(data_np).cuda()
    p_batch = torch.zeros(g.packed_bytes, dtype=torch.uint8, device="cuda")
    p_plain = torch.zeros_like(p_batch)
    torch.cuda.synchronize()
    assert halo.pack_plain(g, data.data_ptr(), p_plain.data_ptr()) == g.packed_bytes
    b = halo.HaloBatch([g], [data.data_ptr()], [p_batch.data_ptr()])
    assert b.nregions == 26
    b.launch()
    torch.cuda.synchronize()
    want = oracle_pack(g, data_np)
    assert p_plain.cpu().numpy().tobytes() == want.tobytes()
    assert p_batch.cpu().numpy().tobytes() == want.tobytes()

    # unpack into ghost cells, batched and plain
    ghost = torch.from_numpy(data_np.copy()).cuda()
    ghost2 = ghost.clone()
    ub = halo.HaloBatch([g], [ghost.data_ptr()], [p_batch.data_ptr()], unpack=True)
    ub.launch()
    halo.unpack_plain(g, p_plain.data_ptr(), ghost2.data_ptr())
    torch.cuda.synchronize()
    exp = oracle_unpack(g, want, data_np)
    assert ghost.cpu().numpy().tobytes() == exp.tobytes()
    assert ghost2.cpu().numpy().tobytes() == exp.tobytes()
    b.close()
    ub.close()


def test_graph_replay_sees_new_data(cuda, mpi_init):
    import torch

    g = halo.Grid((24, 10, 7), 2)
    data = torch.zeros(g.nbytes, dtype=torch.uint8, device="cuda")
    packed = torch.zeros(g.packed_bytes, dtype=torch.uint8, device="cuda")
    s = torch.cuda.Stream()
    b = halo.HaloBatch([g], [data.data_ptr()], [packed.data_ptr()])
    with torch.cuda.stream(s):
        b.capture(s.cuda_stream)
    for seed in (1, 2, 3):
        d_np = H.splitmix_bytes(g.nbytes, seed)
        data.copy_(torch.from_numpy(d_np))
        torch.cuda.synchronize()
        b.replay(s.cuda_stream)
        s.synchronize()
        assert packed.cpu().numpy().tobytes() == oracle_pack(g, d_np).tobytes()
    b.close()


def test_mixed_batch_of_8_grids(cuda, mpi_init):
    """Eight grids with log-uniform interiors and radius 1-3, 208 regions,
    one launch (the mixed halo batch at test sizes)."""
    import torch

    rng = np.random.default_rng(3)
    grids, datas, packs, nps = [], [], [], []
    for i in range(8):
        interior = [int(np.exp(rng.uniform(np.log(4), np.log(24)))) for _ in range(3)]
        g = halo.Grid(interior, int(rng.integers(1, 4)))
        d_np = H.splitmix_bytes(g.nbytes, 50 + i)
        grids.append(g)
        nps.append(d_np)
        datas.append(torch.from_numpy(d_np).cuda())
        packs.append(torch.zeros(g.packed_bytes, dtype=torch.uint8, device="cuda"))
    b = halo.HaloBatch(grids, [d.data_ptr() for d in datas], [p.data_ptr() for p in packs])
    assert b.nregions == 208
    b.launch()
    torch.cuda.synchronize()
    for g, d_np, p in zip(grids, nps, packs):
        assert p.cpu().numpy().tobytes() == oracle_pack(g, d_np).tobytes()
    b.close()


def test_batch_counts_one_launch(cuda, mpi_init):
    import torch

    g = halo.Grid((12, 12, 12), 2)
    data = torch.zeros(g.nbytes, dtype=torch.uint8, device="cuda")
    packed = torch.zeros(g.packed_bytes, dtype=torch.uint8, device="cuda")
    b = halo.HaloBatch([g], [data.data_ptr()], [packed.data_ptr()])
    n0 = _lib.tempi().tempi_kernel_launches()
    b.launch()
    torch.cuda.synchronize()
    assert _lib.tempi().tempi_kernel_launches() == n0 + 1
    n0 = _lib.tempi().tempi_kernel_launches()
    halo.pack_plain(g, data.data_ptr(), packed.data_ptr())
    assert _lib.tempi().tempi_kernel_launches() == n0 + 26
    b.close()


def test_batch_of_1500_regions(cuda, mpi_init):
    """More regions than one warp-search round can cover twice (three rounds
    of the region lookup), each a small strided object of its own."""
    import torch

    rng = np.random.default_rng(9)
    n = 1500
    buf_np = H.splitmix_bytes(n * 256, 77)
    buf = torch.from_numpy(buf_np).cuda()
    regs, wants, offs, pos = [], [], [], 0
    for i in range(n):
        bl = int(rng.integers(1, 9))
        cnt = int(rng.integers(1, 6))
        st = bl + int(rng.integers(0, 8))
        d = _lib.Desc.make(0, st * cnt, bl, [cnt], [st])
        base = i * 256
        o = T.hvector(cnt, 1, st, T.contiguous(bl, T.BYTE))
        wants.append(T.pack(o, buf_np, 1, origin=base))
        offs.append(pos)
        pos += d.size
        regs.append((base, d))
    packed = torch.zeros(pos, dtype=torch.uint8, device="cuda")
    rr = []
    for (base, d), off in zip(regs, offs):
        r = _lib.Region()
        r.origin = buf.data_ptr() + base
        r.packed = packed.data_ptr() + off
        r.desc = d
        r.incount = 1
        rr.append(r)
    import ctypes

    arr = (_lib.Region * n)(*rr)
    h = ctypes.c_void_p()
    _lib.check(_lib.tempi().tempi_batch_create(arr, n, 0, ctypes.byref(h)))
    _lib.check(_lib.tempi().tempi_batch_launch(h, None))
    torch.cuda.synchronize()
    assert packed.cpu().numpy().tobytes() == np.concatenate(wants).tobytes()
    _lib.tempi().tempi_batch_destroy(h)


@pytest.mark.parametrize("unpack", [0, 1])
def test_batch_random_regions(cuda, mpi_init, unpack):
    """One batched launch over 50 seeded random regions (0-3 strided
    dimensions at any alignment, 1-3 objects each, some empty) packing into,
    or unpacking from, one packed buffer at odd offsets: the packed bytes
    equal each region's descriptor oracle in order, and an unpack writes
    exactly the described bytes."""
    import ctypes

    import torch

    from .test_canon import desc_pack
    from .test_exchange_gpu import _rand_desc, desc_unpack

    rng = np.random.default_rng(515 + unpack)
    regs, pos, base = [], 0, 0
    for i in range(50):
        d = _rand_desc(rng, 100000)
        n = 0 if i % 17 == 5 else int(rng.integers(1, 4))
        pos += int(rng.integers(0, 8))
        regs.append((base, d, n, pos))
        pos += d.size * n
        base += d.extent * max(n, 1) + 64
    typed_np = H.splitmix_bytes(base, 99)
    packed_np = H.splitmix_bytes(pos + 64, 98)
    typed = torch.from_numpy(typed_np if not unpack else np.full(base, 0xAA, np.uint8)).cuda()
    packed = torch.from_numpy(packed_np if unpack else np.full(pos + 64, 0x5A, np.uint8)).cuda()
    arr = (_lib.Region * len(regs))()
    for k, (b, d, n, off) in enumerate(regs):
        arr[k].origin = typed.data_ptr() + b
        arr[k].packed = packed.data_ptr() + off
        arr[k].desc = d
        arr[k].incount = n
    h = ctypes.c_void_p()
    _lib.check(_lib.tempi().tempi_batch_create(arr, len(regs), unpack, ctypes.byref(h)))
    _lib.check(_lib.tempi().tempi_batch_launch(h, None))
    torch.cuda.synchronize()
    _lib.tempi().tempi_batch_destroy(h)
    if not unpack:
        want = np.full(pos + 64, 0x5A, np.uint8)
        for b, d, n, off in regs:
            if n:
                want[off: off + d.size * n] = desc_pack(d, typed_np[b:], n)
        assert packed.cpu().numpy().tobytes() == want.tobytes()
    else:
        want = np.full(base, 0xAA, np.uint8)
        for b, d, n, off in regs:
            if n:
                desc_unpack(d, packed_np[off: off + d.size * n], want[b:], n)
        assert typed.cpu().numpy().tobytes() == want.tobytes()


def test_tuned_batch_is_exact_and_remembered(cuda, mpi_init, tmp_path):
    """tempi_batch_tune times launch shapes and per-class chunk passes on the
    batch itself and keeps the fastest: the batch's output stays the oracle's
    (pack and ghost unpack), its choices are reported per region class, and a
    new batch of the same signature starts with them; capture works again
    after tuning.  The tuning file goes to a scratch TEMPI_CACHE_DIR."""
    import os

    import torch

    lib = _lib.tempi()
    old = os.environ.get("TEMPI_CACHE_DIR")
    os.environ["TEMPI_CACHE_DIR"] = str(tmp_path)
    lib.tempi_reload_env()
    try:
        g = halo.Grid((40, 33, 17), 2)
        data_np = H.splitmix_bytes(g.nbytes, 404)
        data = torch.from_numpy(data_np).cuda()
        packed = torch.zeros(g.packed_bytes, dtype=torch.uint8, device="cuda")
        b = halo.HaloBatch([g], [data.data_ptr()], [packed.data_ptr()])
        th0, cps0, cls0 = b.config()
        assert th0 in (128, 256, 512) and set(cls0.values()) <= {1, 2, 4}
        b.tune(None, 2)
        th, cps, cls = b.config()
        assert th in (128, 256, 512) and cps >= 0 and set(cls) == set(cls0)
        assert set(cls.values()) <= {1, 2, 4}
        b.launch()
        torch.cuda.synchronize()
        want = oracle_pack(g, data_np)
        assert packed.cpu().numpy().tobytes() == want.tobytes()
        s = torch.cuda.Stream()
        packed.zero_()
        b.capture(s.cuda_stream)
        b.replay(s.cuda_stream)
        s.synchronize()
        assert packed.cpu().numpy().tobytes() == want.tobytes()
        # a new batch over other buffers with the same regions: same choices
        data2 = torch.from_numpy(H.splitmix_bytes(g.nbytes, 405)).cuda()
        packed2 = torch.zeros_like(packed)
        b2 = halo.HaloBatch([g], [data2.data_ptr()], [packed2.data_ptr()])
        assert b2.config() == (th, cps, cls)
        b2.launch()
        torch.cuda.synchronize()
        assert packed2.cpu().numpy().tobytes() == oracle_pack(g, data2.cpu().numpy()).tobytes()
        assert (tmp_path / "tempi_b200_batch_tune.txt").exists()
        # the tuned unpack into ghost cells
        ghost = data.clone()
        ub = halo.HaloBatch([g], [ghost.data_ptr()], [packed.data_ptr()], unpack=True)
        ub.tune(None, 2)
        ub.launch()
        torch.cuda.synchronize()
        assert ghost.cpu().numpy().tobytes() == oracle_unpack(g, want, data_np).tobytes()
        b.close()
        b2.close()
        ub.close()
    finally:
        if old is None:
            os.environ.pop("TEMPI_CACHE_DIR", None)
        else:
            os.environ["TEMPI_CACHE_DIR"] = old
        lib.tempi_reload_env()


def test_tuned_copy_batch_is_exact(cuda, mpi_init, tmp_path):
    """The fused exchange (a copy batch) tuned the same way still leaves the
    oracle's grid."""
    import os

    import torch

    lib = _lib.tempi()
    old = os.environ.get("TEMPI_CACHE_DIR")
    os.environ["TEMPI_CACHE_DIR"] = str(tmp_path)
    lib.tempi_reload_env()
    try:
        g = halo.Grid((30, 20, 10), 3)
        data_np = H.splitmix_bytes(g.nbytes, 77)
        data = torch.from_numpy(data_np).cuda()
        x = halo.HaloExchange([g], [data.data_ptr()])
        x.tune(None, 2)
        data.copy_(torch.from_numpy(data_np))
        x.launch()
        torch.cuda.synchronize()
        assert data.cpu().numpy().tobytes() == oracle_unpack(g, oracle_pack(g, data_np),
                                                              data_np).tobytes()
        x.close()
    finally:
        if old is None:
            os.environ.pop("TEMPI_CACHE_DIR", None)
        else:
            os.environ["TEMPI_CACHE_DIR"] = old
        lib.tempi_reload_env()
