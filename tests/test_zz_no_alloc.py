"""tempi_batch_run_static: the batched pack for callers that cannot allocate
device memory where they pack (a step of a latency-critical loop, where
cudaMalloc could synchronise the whole device, or an application whose memory
pool already owns the GPU).  It keeps the region table in a fixed array in the
library instead of memory from cudaMalloc.  Checked here against the existing
batched entry point (tempi_batch_create + tempi_batch_launch), byte for byte,
on two calls in a row, and against the descriptor oracle on tables that span
several fill pieces (128 entries each), exactly 1024 regions, and tables whose
last regions are empty.  This file is collected last so that a run stopping at
its first failure has already run every other test; it also passes alone."""
import ctypes

import numpy as np
import pytest

from tempi_b200 import _lib, halo

from . import helpers as H
from .test_canon import desc_pack
from .test_exchange_gpu import _rand_desc, desc_unpack

pytestmark = pytest.mark.gpu


def run_static(regs, unpack, stream=None):
    arr = (_lib.Region * len(regs))(*regs)
    return _lib.tempi().tempi_batch_run_static(arr, len(regs), int(unpack), stream)


def test_static_batch_matches_allocating_batch(cuda, mpi_init):
    import torch

    for call, (interior, radius) in enumerate((((20, 17, 9), 2), ((33, 8, 12), 3))):
        g = halo.Grid(interior, radius)
        data = torch.from_numpy(H.splitmix_bytes(g.nbytes, 100 + call)).cuda()
        want = torch.zeros(g.packed_bytes, dtype=torch.uint8, device="cuda")
        got = torch.full_like(want, 0x55)
        b = halo.HaloBatch([g], [data.data_ptr()], [want.data_ptr()])
        b.launch()
        regs = halo.regions([g], [data.data_ptr()], [got.data_ptr()])
        assert run_static(regs, False) == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert got.cpu().numpy().tobytes() == want.cpu().numpy().tobytes(), call
        # unpack into ghost cells, both ways
        g1 = data.clone()
        g2 = data.clone()
        ub = halo.HaloBatch([g], [g1.data_ptr()], [want.data_ptr()], unpack=True)
        ub.launch()
        uregs = halo.regions([g], [g2.data_ptr()], [got.data_ptr()], unpack=True)
        assert run_static(uregs, True) == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert g1.cpu().numpy().tobytes() == g2.cpu().numpy().tobytes(), call
        b.close()
        ub.close()


def _random_table(rng, n, max_bytes, empty_tail, sparse):
    """n seeded random regions over one typed and one packed buffer; the
    last `empty_tail` regions have no objects, and with `sparse` every 37th
    is empty too."""
    regs, pos, base = [], 0, 0
    for i in range(n):
        d = _rand_desc(rng, max_bytes)
        hole = i >= n - empty_tail or (sparse and i % 37 == 11)
        cnt = 0 if hole else int(rng.integers(1, 3))
        pos += int(rng.integers(0, 8))  # odd gaps between packed regions
        regs.append((base, d, cnt, pos))
        pos += d.size * cnt
        # the last object can reach `start` (< 20) bytes past its extent
        base += d.extent * max(cnt, 1) + 24 + int(rng.integers(0, 16))
    return regs, base + 64, pos + 64


@pytest.mark.parametrize("n,empty_tail,sparse", [(26, 0, True), (104, 3, True), (300, 5, True),
                                                 (260, 4, False), (1024, 0, False)])
@pytest.mark.parametrize("unpack", [0, 1])
def test_static_batch_matches_oracle(cuda, mpi_init, n, empty_tail, sparse, unpack):
    """Tables of 26 regions (one small piece), 104 (one piece, trailing
    empties), 300 (two full pieces and a partial one), 260 (two full pieces,
    then only empty regions) and 1024 (eight full pieces); the packed bytes are
    the descriptor oracle's, region after region, and an unpack writes
    exactly the described bytes (gaps prefilled with 0xAA stay 0xAA).  Two
    calls in a row with different data."""
    import torch

    rng = np.random.default_rng(4000 + n + unpack)
    regs, typed_n, packed_n = _random_table(rng, n, 4000 if n > 300 else 20000, empty_tail,
                                             sparse)
    for call in range(2):
        typed_np = H.splitmix_bytes(typed_n, 10 * n + call)
        packed_np = H.splitmix_bytes(packed_n, 20 * n + call)
        typed = torch.from_numpy(typed_np if not unpack else np.full(typed_n, 0xAA, np.uint8)).cuda()
        packed = torch.from_numpy(packed_np if unpack else np.full(packed_n, 0x5A, np.uint8)).cuda()
        rr = []
        for b, d, cnt, off in regs:
            r = _lib.Region()
            r.origin = typed.data_ptr() + b
            r.packed = packed.data_ptr() + off
            r.desc = d
            r.incount = cnt
            rr.append(r)
        assert run_static(rr, unpack) == 0, _lib.last_error()
        torch.cuda.synchronize()
        if not unpack:
            want = np.full(packed_n, 0x5A, np.uint8)
            for b, d, cnt, off in regs:
                if cnt:
                    want[off: off + d.size * cnt] = desc_pack(d, typed_np[b:], cnt)
            assert packed.cpu().numpy().tobytes() == want.tobytes(), call
        else:
            want = np.full(typed_n, 0xAA, np.uint8)
            for b, d, cnt, off in regs:
                if cnt:
                    desc_unpack(d, packed_np[off: off + d.size * cnt], want[b:], cnt)
            assert typed.cpu().numpy().tobytes() == want.tobytes(), call


def test_static_batch_bad_region_launches_nothing(cuda, mpi_init):
    """A table whose last region is invalid is rejected before anything is
    launched: the output keeps its old bytes."""
    import torch

    g = halo.Grid((6, 5, 4), 1)
    data = torch.from_numpy(H.splitmix_bytes(g.nbytes, 3)).cuda()
    packed = torch.full((g.packed_bytes,), 0x33, dtype=torch.uint8, device="cuda")
    regs = halo.regions([g], [data.data_ptr()], [packed.data_ptr()])
    bad = _lib.Region()
    bad.origin, bad.packed = data.data_ptr(), packed.data_ptr()
    bad.desc = _lib.Desc.make(0, 64, 8, [4], [16])
    bad.desc.ndims = 9  # more dimensions than a descriptor holds
    bad.incount = 1
    n0 = _lib.tempi().tempi_kernel_launches()
    assert run_static(regs + [bad], False) == 1  # TEMPI_ERR_ARG
    torch.cuda.synchronize()
    assert _lib.tempi().tempi_kernel_launches() == n0
    assert bool((packed == 0x33).all())


def test_static_batch_rejects_too_many_regions(cuda, mpi_init):
    import torch

    g = halo.Grid((4, 4, 4), 1)
    data = torch.zeros(g.nbytes, dtype=torch.uint8, device="cuda")
    packed = torch.zeros(g.packed_bytes, dtype=torch.uint8, device="cuda")
    regs = halo.regions([g], [data.data_ptr()], [packed.data_ptr()]) * 40  # 1040 regions
    assert run_static(regs, False) == 1  # TEMPI_ERR_ARG
    assert "at most 1024 regions" in _lib.last_error()
