"""One rank of a multi-process test (tests/test_ranks.py, tests/test_ranks_gpu.py):
``python -m tests.ranks_worker <scenario> [device]``, started once per rank with
MINIMPI_SIZE, MINIMPI_RANK and MINIMPI_DIR set, so the stand-in MPI library
joins the ranks over Unix sockets.  Each scenario checks its own results
against the oracle and raises on a mismatch; the process exits 0 on success.
With ``device`` the buffers live in GPU memory (every rank on cuda:0; the
ranks wait for each other only on the host)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import types as T  # noqa: E402
from tempi_b200 import _lib, halo, mpi  # noqa: E402


def seeded(n, seed):
    return np.random.default_rng(seed).integers(0, 256, n, dtype=np.uint8)


class Bufs:
    """Host numpy arrays, or device tensors, behind one interface."""

    def __init__(self, device):
        self.device = device
        if device:
            import torch

            self.torch = torch

    def put(self, a):
        if not self.device:
            return np.ascontiguousarray(a)
        return self.torch.from_numpy(np.ascontiguousarray(a)).cuda()

    def ptr(self, b):
        return b.data_ptr() if self.device else b.ctypes.data

    def get(self, b):
        if not self.device:
            return b
        self.torch.cuda.synchronize()
        return b.cpu().numpy()


def p2p(rank, size, bufs):
    """A ring of strided messages, tags per sender, an MPI_ANY_SOURCE
    receive, and two 8 MiB messages crossing at once (both ranks send before
    either receives)."""
    right, left = (rank + 1) % size, (rank - 1) % size
    t = mpi.Type_vector(64, 8, 16, mpi.BYTE)
    assert mpi.Type_commit(t) == 0
    o = T.vector(64, 8, 16, T.BYTE)
    methods = ["DEVICE", "ONESHOT", "STAGED"] if bufs.device else [None]
    for m in methods:
        if m:
            for k in ("DEVICE", "ONESHOT", "STAGED"):
                os.environ.pop("TEMPI_DATATYPE_" + k, None)
            os.environ["TEMPI_DATATYPE_" + m] = ""
            _lib.tempi().tempi_reload_env()
        mine = seeded(o.extent, 10 * rank + 1)
        src = bufs.put(mine)
        dst = bufs.put(np.full(o.extent, 0xAA, np.uint8))
        err, rq = mpi.Irecv(bufs.ptr(dst), 1, t, source=left, tag=left)
        assert err == 0, _lib.last_error()
        err, sq = mpi.Isend(bufs.ptr(src), 1, t, dest=right, tag=rank)
        assert err == 0, _lib.last_error()
        assert mpi.Wait(sq)[0] == 0 and mpi.Wait(rq)[0] == 0, _lib.last_error()
        exp = np.full(o.extent, 0xAA, np.uint8)
        T.unpack(o, T.pack(o, seeded(o.extent, 10 * left + 1), 1), exp, 1)
        assert bufs.get(dst).tobytes() == exp.tobytes(), (m, rank)
        # blocking send / receive the other way round
        if rank % 2 == 0:
            assert mpi.Send(bufs.ptr(src), 1, t, dest=left, tag=99) == 0
            err, _ = mpi.Recv(bufs.ptr(dst), 1, t, source=right, tag=99)
        else:
            err, _ = mpi.Recv(bufs.ptr(dst), 1, t, source=right, tag=99)
            assert err == 0
            err = mpi.Send(bufs.ptr(src), 1, t, dest=left, tag=99)
        assert err == 0, _lib.last_error()
        exp = np.full(o.extent, 0xAA, np.uint8)
        T.unpack(o, T.pack(o, seeded(o.extent, 10 * right + 1), 1), exp, 1)
        assert bufs.get(dst).tobytes() == exp.tobytes(), (m, rank, "blocking")
    for k in ("DEVICE", "ONESHOT", "STAGED"):
        os.environ.pop("TEMPI_DATATYPE_" + k, None)
    _lib.tempi().tempi_reload_env()
    # any source: rank 0 gathers one message from every other rank
    if rank == 0:
        got = set()
        for _ in range(size - 1):
            buf = np.zeros(4, np.int32)
            err, st = mpi.Recv(buf.ctypes.data, 4, mpi.INT, source=mpi.ANY_SOURCE, tag=7)
            assert err == 0
            got.add(int(buf[0]))
        assert got == set(range(1, size))
    else:
        buf = np.full(4, rank, np.int32)
        assert mpi.Send(buf.ctypes.data, 4, mpi.INT, dest=0, tag=7) == 0
    # large messages crossing: each rank sends 8 MiB to its right before it
    # receives from its left (the library must read while it writes)
    n = 8 << 20
    big = seeded(n, 500 + rank)
    out = np.zeros(n, np.uint8)
    err, rq = mpi.Irecv(out.ctypes.data, n, mpi.BYTE, source=left, tag=5)
    assert err == 0
    assert mpi.Send(big.ctypes.data, n, mpi.BYTE, dest=right, tag=5) == 0
    assert mpi.Wait(rq)[0] == 0
    assert out.tobytes() == seeded(n, 500 + left).tobytes()
    mpi.Type_free(t)


def _grid_data(g, rank):
    return seeded(g.nbytes, 2000 + rank)


def _expected_grid(g, rank, size, nbr):
    """This rank's grid after a periodic halo exchange in which direction d's
    send region of rank nbr(r, d) lands in ghost region -d of rank r."""
    sizes = [g.alloc[2], g.alloc[1], g.alloc[0]]
    exp = _grid_data(g, rank).copy()
    for d in halo.directions():
        src = nbr(rank, tuple(-x for x in d))
        subs, starts = g.region_shape[(d, False)]
        data = T.pack(T.subarray(sizes, subs, starts, T.ORDER_C, T.DOUBLE),
                      _grid_data(g, src), 1)
        subs, starts = g.region_shape[(tuple(-x for x in d), True)]
        T.unpack(T.subarray(sizes, subs, starts, T.ORDER_C, T.DOUBLE), data, exp, 1)
    return exp


def _report_regions(g, got, exp, rank, size, nbr):
    """Which ghost regions differ from the oracle, and whose data they hold."""
    sizes = [g.alloc[2], g.alloc[1], g.alloc[0]]

    def region(buf, d, ghost):
        subs, starts = g.region_shape[(d, ghost)]
        return T.pack(T.subarray(sizes, subs, starts, T.ORDER_C, T.DOUBLE), buf, 1)

    for d in halo.directions():
        a, b = region(got, d, True), region(exp, d, True)
        if a.tobytes() == b.tobytes():
            continue
        whose = [(r, e) for r in range(size) for e in halo.directions()
                 if region(_grid_data(g, r), e, False).tobytes() == a.tobytes()]
        print(f"rank {rank}: ghost {d} wrong; holds send region of {whose[:3]}; "
              f"{int((a != b).sum())} of {a.size} bytes differ", flush=True)
    inner = [(d, region(got, d, False).tobytes() == region(exp, d, False).tobytes())
             for d in halo.directions()]
    print(f"rank {rank}: interior send regions intact: {all(x for _, x in inner)}", flush=True)


def halo_exchange(rank, size, bufs):
    """A 3-D grid per rank, the ranks a periodic ring along x (y and z wrap
    onto the rank itself): the interposed MPI_Neighbor_alltoallw over a
    26-edge graph communicator, and the reference's sequence (26 MPI_Pack,
    MPI_Neighbor_alltoallv of the packed bytes, 26 MPI_Unpack), each leaving
    the oracle's grid on every rank."""
    g = halo.Grid((12, 10, 8), 2)

    def nbr(r, d):
        return (r + d[0]) % size

    dirs = halo.directions()
    dests = [nbr(rank, d) for d in dirs]
    sources = [nbr(rank, tuple(-x for x in d)) for d in dirs]
    err, comm = mpi.Dist_graph_create_adjacent(sources, dests)
    assert err == 0
    exp = _expected_grid(g, rank, size, nbr)
    n = len(dirs)
    sendtypes = [g.send[d] for d in dirs]
    recvtypes = [g.recv[tuple(-x for x in d)] for d in dirs]
    # 1. MPI_Neighbor_alltoallw, typed regions in, typed regions out
    grid = bufs.put(_grid_data(g, rank))
    isir0 = _lib.counter("neighbor_isir")
    err = mpi.Neighbor_alltoallw(bufs.ptr(grid), [1] * n, [0] * n, sendtypes, bufs.ptr(grid),
                                 [1] * n, [0] * n, recvtypes, comm)
    assert err == 0, _lib.last_error()
    got = bufs.get(grid)
    if got.tobytes() != exp.tobytes():
        _report_regions(g, got, exp, rank, size, nbr)
    assert got.tobytes() == exp.tobytes(), "alltoallw"
    if bufs.device and size > 1:
        assert _lib.counter("neighbor_isir") == isir0 + 1  # edges to another rank
    # 2. the reference's sequence through MPI_Pack / MPI_Neighbor_alltoallv /
    # MPI_Unpack, packed bytes in between
    grid = bufs.put(_grid_data(g, rank))
    sendbuf = bufs.put(np.zeros(g.packed_bytes, np.uint8))
    recvbuf = bufs.put(np.zeros(g.packed_bytes, np.uint8))
    offs = g.offsets()
    counts = [g.region_bytes[d] for d in dirs]
    displs = [offs[d] for d in dirs]
    assert halo.pack_plain(g, bufs.ptr(grid), bufs.ptr(sendbuf)) == g.packed_bytes
    err = mpi.Neighbor_alltoallv(bufs.ptr(sendbuf), counts, displs, mpi.BYTE,
                                 bufs.ptr(recvbuf), counts, displs, mpi.BYTE, comm)
    assert err == 0
    halo.unpack_plain(g, bufs.ptr(recvbuf), bufs.ptr(grid))
    assert bufs.get(grid).tobytes() == exp.tobytes(), "pack/alltoallv/unpack"
    mpi.Comm_free(comm)


def alltoallv(rank, size, bufs):
    """MPI_Alltoallv of doubles with uneven blocks and gaps between them,
    through the interposer, by every method (device buffers) or the library
    (host buffers): every received block is the sender's, and the gap bytes
    of the receive buffer keep their 0xAA."""
    methods = (["STAGED", "REMOTE_FIRST", "ISIR_STAGED", "ISIR_REMOTE_STAGED", "NONE"]
               if bufs.device else [None])
    def cnt(a, b):  # doubles rank a sends rank b
        return 3 + (5 * a + 7 * b) % 11

    sendcounts = [cnt(rank, j) for j in range(size)]
    recvcounts = [cnt(i, rank) for i in range(size)]
    sdispls, rdispls, pos = [], [], 0
    for c in sendcounts:
        sdispls.append(pos)
        pos += c + 2  # two doubles of gap after every block
    send_n = pos
    pos = 0
    for c in recvcounts:
        rdispls.append(pos)
        pos += c + 1
    recv_n = pos
    send_np = seeded(8 * send_n, 3000 + rank)
    for m in methods:
        for k in ("STAGED", "REMOTE_FIRST", "ISIR_STAGED", "ISIR_REMOTE_STAGED"):
            os.environ.pop("TEMPI_ALLTOALLV_" + k, None)
        os.environ.pop("TEMPI_NO_ALLTOALLV", None)
        if m == "NONE":
            os.environ["TEMPI_NO_ALLTOALLV"] = ""
        elif m:
            os.environ["TEMPI_ALLTOALLV_" + m] = ""
        if m == "ISIR_REMOTE_STAGED":
            os.environ["TEMPI_RANKS_PER_NODE"] = "1"  # every other rank is remote
        else:
            os.environ.pop("TEMPI_RANKS_PER_NODE", None)
        _lib.tempi().tempi_reload_env()
        sendbuf = bufs.put(send_np)
        recvbuf = bufs.put(np.full(8 * recv_n, 0xAA, np.uint8))
        err = mpi.Alltoallv(bufs.ptr(sendbuf), sendcounts, sdispls, mpi.DOUBLE,
                            bufs.ptr(recvbuf), recvcounts, rdispls, mpi.DOUBLE)
        assert err == 0, (m, _lib.last_error())
        got = bufs.get(recvbuf)
        exp = np.full(8 * recv_n, 0xAA, np.uint8)
        for i in range(size):
            # rank i's block for this rank, as rank i laid it out
            other = seeded(8 * send_n_of(i, size, cnt), 3000 + i)
            sd = sdispls_of(i, size, cnt)
            a = 8 * sd[rank]
            exp[8 * rdispls[i]: 8 * (rdispls[i] + recvcounts[i])] = \
                other[a: a + 8 * recvcounts[i]]
        assert got.tobytes() == exp.tobytes(), m
    for k in ("STAGED", "REMOTE_FIRST", "ISIR_STAGED", "ISIR_REMOTE_STAGED"):
        os.environ.pop("TEMPI_ALLTOALLV_" + k, None)
    os.environ.pop("TEMPI_NO_ALLTOALLV", None)
    os.environ.pop("TEMPI_RANKS_PER_NODE", None)
    _lib.tempi().tempi_reload_env()


def sdispls_of(r, size, cnt):
    out, pos = [], 0
    for j in range(size):
        out.append(pos)
        pos += cnt(r, j) + 2
    return out


def send_n_of(r, size, cnt):
    return sum(cnt(r, j) + 2 for j in range(size))


SCENARIOS = {"p2p": p2p, "halo": halo_exchange, "alltoallv": alltoallv}


def main():
    scenario = sys.argv[1]
    device = len(sys.argv) > 2 and sys.argv[2] == "device"
    if device:
        import torch

        torch.cuda.set_device(0)
    assert mpi.Init() == 0
    rank, size = mpi.Comm_rank(), mpi.Comm_size()
    assert size == int(os.environ["MINIMPI_SIZE"]) and rank == int(os.environ["MINIMPI_RANK"])
    SCENARIOS[scenario](rank, size, Bufs(device))
    assert mpi.Barrier() == 0
    assert mpi.Finalize() == 0
    print(f"rank {rank} of {size}: {scenario} ok", flush=True)


if __name__ == "__main__":
    main()
