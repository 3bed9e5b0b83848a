"""tempi_batch_run_static: the batched pack for callers that cannot allocate
device memory where they pack (a step of a latency-critical loop, where
cudaMalloc could synchronise the whole device, or an application whose memory
pool already owns the GPU).  It keeps the region table in a fixed array in the
library instead of memory from cudaMalloc.  Checked here against the existing
batched entry point (tempi_batch_create + tempi_batch_launch), byte for byte,
on two calls in a row.  This file is collected last so that a run stopping at
its first failure has already run every other test; it also passes alone."""
import ctypes

import numpy as np
import pytest

from tempi_b200 import _lib, halo

from . import helpers as H

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


def test_static_batch_rejects_too_many_regions(cuda, mpi_init):
    import torch

    g = halo.Grid((4, 4, 4), 1)
    data = torch.zeros(g.nbytes, dtype=torch.uint8, device="cuda")
    packed = torch.zeros(g.packed_bytes, dtype=torch.uint8, device="cuda")
    regs = halo.regions([g], [data.data_ptr()], [packed.data_ptr()]) * 40  # 1040 regions
    assert run_static(regs, False) == 1  # TEMPI_ERR_ARG
    assert "at most 1024 regions" in _lib.last_error()
