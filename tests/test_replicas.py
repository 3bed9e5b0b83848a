"""The N > 1 path of bench.py is replicas: one process per GPU, each with
its own MPI world of size 1 and its own TEMPI, timed as the max over ranks.
Covered here with two gloo ranks on CPU: each rank runs the interposer on
host buffers independently and the per-rank times reduce to their max."""
import os
import sys

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from oracle import types as T
        from tempi_b200 import mpi

        assert mpi.Init() == 0
        t = mpi.Type_vector(64 + rank, 8, 24, mpi.BYTE)  # a different object per rank
        assert mpi.Type_commit(t) == 0
        src = np.random.default_rng(rank).integers(0, 256, 24 * 80, dtype=np.uint8)
        out = np.zeros(8 * (64 + rank), np.uint8)
        err, pos = mpi.Pack(src.ctypes.data, 1, t, out.ctypes.data, out.nbytes)
        ok = err == 0 and out.tobytes() == T.pack(T.vector(64 + rank, 8, 24, T.BYTE), src, 1).tobytes()
        m = bench.reduce_max(1.5 + rank, dist)
        q.put((rank, ok, m))
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas_reduce_to_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(0, True, 2.5), (1, True, 2.5)]
