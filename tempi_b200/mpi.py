"""Python mirror of the MPI calls on the interposed path.

Each function calls the C entry point of the same name: the interposed ones
(``Type_commit``, ``Type_free``, ``Pack``, ``Unpack``, ``Send``, ``Recv``,
``Isend``, ``Irecv``, ``Wait``, ``Init``, ``Finalize``) through
libtempi_b200.so, the rest (type constructors and queries) through the
underlying MPI library.  Buffers are raw addresses (``tensor.data_ptr()``,
``array.ctypes.data``).  Every call returns what the C call returns; the
ones that fill output arguments return them as a tuple after the error code.
"""
from __future__ import annotations

import ctypes

from . import _lib

# handles and constants of libminimpi's mpi.h
SUCCESS = 0
ERR_TYPE = 3
ERR_ARG = 12
ERR_TRUNCATE = 15
ERR_OTHER = 16
COMM_WORLD = 1
BYTE, CHAR, UNSIGNED_CHAR, SHORT, INT, UNSIGNED, LONG, LONG_LONG = 1, 2, 3, 4, 5, 6, 7, 8
FLOAT, DOUBLE, PACKED = 9, 10, 11
ORDER_C, ORDER_FORTRAN = 56, 57
REQUEST_NULL = 0
ANY_SOURCE, ANY_TAG = -2, -1

_initialized = False


def _ints(xs):
    return (ctypes.c_int * len(xs))(*xs)


def _aints(xs):
    return (ctypes.c_ssize_t * len(xs))(*xs)


def Init() -> int:
    """MPI_Init through the interposer (idempotent for the test process)."""
    global _initialized
    if _initialized:
        return SUCCESS
    err = _lib.tempi().MPI_Init(None, None)
    _initialized = err == SUCCESS
    return err


def Finalize() -> int:
    global _initialized
    _initialized = False
    return _lib.tempi().MPI_Finalize()


def _new(fn, *args):
    out = ctypes.c_int(0)
    err = fn(*args, ctypes.byref(out))
    if err:
        raise RuntimeError(f"{fn.__name__} failed with MPI error {err}")
    return out.value


def Type_contiguous(count, old):
    return _new(_lib.minimpi().MPI_Type_contiguous, count, old)


def Type_vector(count, bl, stride, old):
    return _new(_lib.minimpi().MPI_Type_vector, count, bl, stride, old)


def Type_create_hvector(count, bl, stride, old):
    return _new(_lib.minimpi().MPI_Type_create_hvector, count, bl, stride, old)


def Type_indexed(bls, displs, old):
    return _new(_lib.minimpi().MPI_Type_indexed, len(bls), _ints(bls), _ints(displs), old)


def Type_create_hindexed(bls, displs, old):
    return _new(
        _lib.minimpi().MPI_Type_create_hindexed, len(bls), _ints(bls), _aints(displs), old
    )


def Type_create_indexed_block(bl, displs, old):
    return _new(
        _lib.minimpi().MPI_Type_create_indexed_block, len(displs), bl, _ints(displs), old
    )


def Type_create_hindexed_block(bl, displs, old):
    return _new(
        _lib.minimpi().MPI_Type_create_hindexed_block, len(displs), bl, _aints(displs), old
    )


def Type_create_struct(bls, displs, types):
    return _new(
        _lib.minimpi().MPI_Type_create_struct, len(bls), _ints(bls), _aints(displs),
        _ints(types),
    )


def Type_create_subarray(sizes, subsizes, starts, order, old):
    return _new(
        _lib.minimpi().MPI_Type_create_subarray, len(sizes), _ints(sizes),
        _ints(subsizes), _ints(starts), order, old,
    )


def Type_create_resized(old, lb, extent):
    return _new(_lib.minimpi().MPI_Type_create_resized, old, lb, extent)


def Type_dup(old):
    return _new(_lib.minimpi().MPI_Type_dup, old)


def Type_commit(t: int) -> int:
    h = ctypes.c_int(t)
    err = _lib.tempi().MPI_Type_commit(ctypes.byref(h))
    return err


def Type_free(t: int) -> int:
    h = ctypes.c_int(t)
    return _lib.tempi().MPI_Type_free(ctypes.byref(h))


def Type_size(t: int) -> int:
    return _new(_lib.minimpi().MPI_Type_size, t)


def Type_get_extent(t: int):
    lb, ext = ctypes.c_ssize_t(0), ctypes.c_ssize_t(0)
    err = _lib.minimpi().MPI_Type_get_extent(t, ctypes.byref(lb), ctypes.byref(ext))
    if err:
        raise RuntimeError(f"MPI_Type_get_extent failed with {err}")
    return lb.value, ext.value


def Pack_size(incount: int, t: int) -> int:
    out = ctypes.c_int(0)
    err = _lib.minimpi().MPI_Pack_size(incount, t, COMM_WORLD, ctypes.byref(out))
    if err:
        raise RuntimeError(f"MPI_Pack_size failed with {err}")
    return out.value


def Pack(inbuf: int, incount: int, t: int, outbuf: int, outsize: int,
         position: int = 0, library: bool = False):
    """MPI_Pack; returns (err, new position).  ``library=True`` calls the
    underlying MPI directly, bypassing TEMPI."""
    pos = ctypes.c_int(position)
    lib = _lib.minimpi() if library else _lib.tempi()
    err = lib.MPI_Pack(inbuf, incount, t, outbuf, outsize, ctypes.byref(pos), COMM_WORLD)
    return err, pos.value


def Unpack(inbuf: int, insize: int, outbuf: int, outcount: int, t: int,
           position: int = 0, library: bool = False):
    pos = ctypes.c_int(position)
    lib = _lib.minimpi() if library else _lib.tempi()
    err = lib.MPI_Unpack(inbuf, insize, ctypes.byref(pos), outbuf, outcount, t, COMM_WORLD)
    return err, pos.value


def Send(buf: int, count: int, t: int, dest: int = 0, tag: int = 0) -> int:
    return _lib.tempi().MPI_Send(buf, count, t, dest, tag, COMM_WORLD)


def Recv(buf: int, count: int, t: int, source: int = 0, tag: int = 0):
    st = _lib.Status()
    err = _lib.tempi().MPI_Recv(buf, count, t, source, tag, COMM_WORLD, ctypes.byref(st))
    return err, st


def Isend(buf: int, count: int, t: int, dest: int = 0, tag: int = 0):
    req = ctypes.c_int(0)
    err = _lib.tempi().MPI_Isend(buf, count, t, dest, tag, COMM_WORLD, ctypes.byref(req))
    return err, req.value


def Irecv(buf: int, count: int, t: int, source: int = 0, tag: int = 0):
    req = ctypes.c_int(0)
    err = _lib.tempi().MPI_Irecv(buf, count, t, source, tag, COMM_WORLD, ctypes.byref(req))
    return err, req.value


def Wait(req: int):
    r = ctypes.c_int(req)
    st = _lib.Status()
    err = _lib.tempi().MPI_Wait(ctypes.byref(r), ctypes.byref(st))
    return err, r.value, st


def Get_count(st, t: int) -> int:
    out = ctypes.c_int(0)
    _lib.minimpi().MPI_Get_count(ctypes.byref(st), t, ctypes.byref(out))
    return out.value


def Dist_graph_create_adjacent(sources, destinations, weighted=False):
    """A distributed graph communicator over MPI_COMM_WORLD (MPI-3.1 7.5.4);
    returns (err, comm)."""
    src = (ctypes.c_int * max(len(sources), 1))(*sources)
    dst = (ctypes.c_int * max(len(destinations), 1))(*destinations)
    if weighted:
        sw = (ctypes.c_int * max(len(sources), 1))(*([1] * len(sources)))
        dw = (ctypes.c_int * max(len(destinations), 1))(*([1] * len(destinations)))
    else:
        sw = dw = ctypes.c_void_p(1)  # MPI_UNWEIGHTED
    comm = ctypes.c_int(0)
    err = _lib.minimpi().MPI_Dist_graph_create_adjacent(
        COMM_WORLD, len(sources), src, sw, len(destinations), dst, dw, 0, 0,
        ctypes.byref(comm))
    return err, comm.value


def Comm_free(comm: int) -> int:
    c = ctypes.c_int(comm)
    return _lib.minimpi().MPI_Comm_free(ctypes.byref(c))


def _ints(v):
    return (ctypes.c_int * max(len(v), 1))(*[int(x) for x in v])


def _aints(v):
    return (ctypes.c_ssize_t * max(len(v), 1))(*[int(x) for x in v])


def Neighbor_alltoallv(sendbuf: int, sendcounts, sdispls, sendtype: int, recvbuf: int,
                       recvcounts, rdispls, recvtype: int, comm: int) -> int:
    """MPI_Neighbor_alltoallv: not interposed (the reference forwards it
    unchanged), so this is the library's."""
    return _lib.minimpi().MPI_Neighbor_alltoallv(
        sendbuf, _ints(sendcounts), _ints(sdispls), sendtype, recvbuf, _ints(recvcounts),
        _ints(rdispls), recvtype, comm)


def Neighbor_alltoallw(sendbuf: int, sendcounts, sdispls, sendtypes, recvbuf: int,
                       recvcounts, rdispls, recvtypes, comm: int,
                       library: bool = False) -> int:
    """MPI_Neighbor_alltoallw; displacements in bytes.  ``library=True``
    calls the underlying MPI directly."""
    lib = _lib.minimpi() if library else _lib.tempi()
    return lib.MPI_Neighbor_alltoallw(
        sendbuf, _ints(sendcounts), _aints(sdispls), _ints(sendtypes), recvbuf,
        _ints(recvcounts), _aints(rdispls), _ints(recvtypes), comm)


def Alltoallv(sendbuf: int, sendcounts, sdispls, sendtype: int, recvbuf: int, recvcounts,
              rdispls, recvtype: int, comm: int = None, library: bool = False) -> int:
    """MPI_Alltoallv; displacements in extents of the types.  ``library=True``
    calls the underlying MPI directly."""
    lib = _lib.minimpi() if library else _lib.tempi()
    return lib.MPI_Alltoallv(sendbuf, _ints(sendcounts), _ints(sdispls), sendtype, recvbuf,
                             _ints(recvcounts), _ints(rdispls), recvtype,
                             COMM_WORLD if comm is None else comm)


def Comm_rank(comm: int = None) -> int:
    out = ctypes.c_int(0)
    err = _lib.minimpi().MPI_Comm_rank(COMM_WORLD if comm is None else comm, ctypes.byref(out))
    if err:
        raise RuntimeError(f"MPI_Comm_rank failed with {err}")
    return out.value


def Comm_size(comm: int = None) -> int:
    out = ctypes.c_int(0)
    err = _lib.minimpi().MPI_Comm_size(COMM_WORLD if comm is None else comm, ctypes.byref(out))
    if err:
        raise RuntimeError(f"MPI_Comm_size failed with {err}")
    return out.value


def Barrier(comm: int = None) -> int:
    return _lib.minimpi().MPI_Barrier(COMM_WORLD if comm is None else comm)


def describe(t: int):
    """TEMPI's canonical strided block for a type (tempi_describe)."""
    d = _lib.Desc()
    err = _lib.tempi().tempi_describe(t, ctypes.byref(d))
    return err, d
