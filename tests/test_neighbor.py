"""Neighbourhood collectives on a distributed graph communicator, with host
buffers (CPU): the self-only library's MPI_Neighbor_alltoallv and
MPI_Neighbor_alltoallw, and the interposed MPI_Neighbor_alltoallw on its
library and Isend/Irecv paths.  In a world of one rank every edge is a
self-edge; the k-th out-edge meets the k-th in-edge."""
import numpy as np

from oracle import types as T
from tempi_b200 import _lib, mpi

from . import helpers as H


def test_graph_counts_and_free(mpi_init):
    err, comm = mpi.Dist_graph_create_adjacent([0, 0, 0], [0, 0])
    assert err == 0 and comm not in (0, mpi.COMM_WORLD)
    import ctypes

    i, o, w = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    assert _lib.minimpi().MPI_Dist_graph_neighbors_count(comm, ctypes.byref(i), ctypes.byref(o),
                                                         ctypes.byref(w)) == 0
    assert (i.value, o.value, w.value) == (3, 2, 0)
    assert mpi.Comm_free(comm) == 0
    assert mpi.Comm_free(comm) != 0  # already freed
    err, _ = mpi.Dist_graph_create_adjacent([1], [0])  # no rank 1 in this world
    assert err != 0


def test_neighbor_alltoallv_bytes_match_edges_in_order(mpi_init):
    err, comm = mpi.Dist_graph_create_adjacent([0, 0, 0], [0, 0, 0])
    assert err == 0
    send = np.arange(100, dtype=np.uint8)
    recv = np.full(100, 0xAA, np.uint8)
    counts, sd, rd = [10, 20, 30], [0, 10, 30], [70, 40, 0]
    assert mpi.Neighbor_alltoallv(send.ctypes.data, counts, sd, mpi.BYTE, recv.ctypes.data,
                                  counts, rd, mpi.BYTE, comm) == 0
    want = np.full(100, 0xAA, np.uint8)
    for c, s, r in zip(counts, sd, rd):
        want[r:r + c] = send[s:s + c]
    assert recv.tobytes() == want.tobytes()
    mpi.Comm_free(comm)


def halo_types():
    """Send and receive regions of a small periodic grid of doubles (interior
    4x5x6, radius 1; sizes listed slowest first): two faces and an edge, each
    send region paired with the ghost region on the opposite side."""
    sizes = [6, 7, 8]
    d = H.named("DOUBLE")
    sub = lambda s, st: H.subarray(sizes, s, st, mpi.ORDER_C, d)
    send = [sub([4, 5, 1], [1, 1, 6]),   # +x face
            sub([4, 1, 6], [1, 5, 1]),   # +y face
            sub([1, 1, 6], [4, 5, 1])]   # +y+z edge
    recv = [sub([4, 5, 1], [1, 1, 0]),   # -x ghost
            sub([4, 1, 6], [1, 0, 1]),   # -y ghost
            sub([1, 1, 6], [0, 0, 1])]   # -y-z ghost
    return sizes, send, recv


def test_neighbor_alltoallw_host_library_and_interposed(mpi_init):
    sizes, st, rt = halo_types()
    nbytes = int(np.prod(sizes)) * 8
    grid = H.splitmix_bytes(nbytes, 5)
    want = grid.copy()
    for a, b in zip(st, rt):
        T.unpack(b.o, T.pack(a.o, grid, 1), want, 1)
    for t in st + rt:
        t.commit()
    for library in (True, False):
        g = grid.copy()
        err, comm = mpi.Dist_graph_create_adjacent([0, 0, 0], [0, 0, 0])
        assert err == 0
        before = {k: _lib.counter(k) for k in ("neighbor_fused", "neighbor_isir", "neighbor_lib")}
        assert mpi.Neighbor_alltoallw(g.ctypes.data, [1, 1, 1], [0, 0, 0], [t.h for t in st],
                                      g.ctypes.data, [1, 1, 1], [0, 0, 0], [t.h for t in rt],
                                      comm, library=library) == 0
        assert g.tobytes() == want.tobytes(), library
        if not library:  # host buffers: TEMPI sends them the reference's way
            assert _lib.counter("neighbor_isir") == before["neighbor_isir"] + 1
        mpi.Comm_free(comm)
