"""Loads the native libraries and declares their C signatures.

``libtempi_b200.so`` (the interposer and its kernels) is loaded globally
first and ``libminimpi.so`` (the self-only MPI library standing in for the
system MPI) after it: the order an application gets by linking
``-ltempi_b200 -lmpi``.  Any library loaded later that calls MPI_Pack binds
to the interposer, and the interposer reaches the library's MPI_Pack with
dlsym(RTLD_NEXT).  Calls through ``minimpi()`` reach the underlying library
directly.

There is no fallback: if a library is missing this raises, telling the user
to build it.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
MINIMPI_SO = os.path.join(CSRC, "libminimpi.so")
TEMPI_SO = os.path.join(CSRC, "libtempi_b200.so")

TEMPI_MAX_DIMS = 4

c_int, c_int64, c_void_p = ctypes.c_int, ctypes.c_int64, ctypes.c_void_p
P = ctypes.POINTER


class Desc(ctypes.Structure):
    """``tempi_desc`` (include/tempi_b200.h)."""

    _fields_ = [
        ("start", c_int64),
        ("extent", c_int64),
        ("block", c_int64),
        ("size", c_int64),
        ("ndims", ctypes.c_int32),
        ("align", ctypes.c_int32),
        ("counts", c_int64 * TEMPI_MAX_DIMS),
        ("strides", c_int64 * TEMPI_MAX_DIMS),
    ]

    def as_dict(self):
        n = self.ndims
        return dict(
            start=self.start, extent=self.extent, block=self.block, size=self.size,
            ndims=n, align=self.align, counts=list(self.counts[:n]),
            strides=list(self.strides[:n]),
        )

    @classmethod
    def make(cls, start, extent, block, counts, strides, align=None):
        d = cls()
        d.start, d.extent, d.block = start, extent, block
        d.ndims = len(counts)
        size = block
        for k, (c, s) in enumerate(zip(counts, strides)):
            d.counts[k] = c
            d.strides[k] = s
            size *= c
        d.size = size
        if align is None:
            bits = start | block | extent
            for s in strides:
                bits |= s & 0xFFFFFFFFFFFFFFFF
            align = 16
            while align > 1 and bits & (align - 1):
                align >>= 1
        d.align = align
        return d


class Config(ctypes.Structure):
    """``tempi_config``."""

    _fields_ = [
        ("kernel", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("threads", ctypes.c_int32),
        ("unroll", ctypes.c_int32),
        ("blocks_per_sm", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


# The cost model's ten kernel configurations, in the order of its outputs
# (kCandidates in csrc/tempi/dispatch.cpp): word kernel at 256, 512 and 128
# threads; row kernel; shift kernel at 4, 8, 16, 32 lanes per row; staged
# kernel at 3 and 8 CTAs per SM.
CANDIDATE_CONFIGS = (
    (1, 0, 256, 0, 0, 0), (1, 0, 512, 0, 0, 0), (1, 0, 128, 0, 0, 0),
    (2, 0, 256, 0, 0, 0),
    (3, 0, 256, 4, 0, 0), (3, 0, 256, 8, 0, 0), (3, 0, 256, 16, 0, 0), (3, 0, 256, 32, 0, 0),
    (4, 0, 256, 0, 3, 0), (4, 0, 256, 0, 8, 0),
)


class Region(ctypes.Structure):
    """``tempi_region``."""

    _fields_ = [
        ("origin", c_void_p),
        ("packed", c_void_p),
        ("desc", Desc),
        ("incount", c_int64),
    ]


class CopyRegion(ctypes.Structure):
    """``tempi_copy_region``."""

    _fields_ = [
        ("src_origin", c_void_p),
        ("dst_origin", c_void_p),
        ("src_desc", Desc),
        ("dst_desc", Desc),
        ("src_count", c_int64),
        ("dst_count", c_int64),
    ]


class Status(ctypes.Structure):
    """``MPI_Status`` of libminimpi's mpi.h."""

    _fields_ = [
        ("MPI_SOURCE", c_int),
        ("MPI_TAG", c_int),
        ("MPI_ERROR", c_int),
        ("reserved_", c_int),
        ("bytes_", ctypes.c_longlong),
    ]


_minimpi = None
_tempi = None

_MPI_SIGS = {
    "MPI_Init": (c_int, [c_void_p, c_void_p]),
    "MPI_Init_thread": (c_int, [c_void_p, c_void_p, c_int, P(c_int)]),
    "MPI_Finalize": (c_int, []),
    "MPI_Initialized": (c_int, [P(c_int)]),
    "MPI_Comm_rank": (c_int, [c_int, P(c_int)]),
    "MPI_Comm_size": (c_int, [c_int, P(c_int)]),
    "MPI_Type_contiguous": (c_int, [c_int, c_int, P(c_int)]),
    "MPI_Type_vector": (c_int, [c_int, c_int, c_int, c_int, P(c_int)]),
    "MPI_Type_create_hvector": (c_int, [c_int, c_int, ctypes.c_ssize_t, c_int, P(c_int)]),
    "MPI_Type_indexed": (c_int, [c_int, P(c_int), P(c_int), c_int, P(c_int)]),
    "MPI_Type_create_hindexed": (c_int, [c_int, P(c_int), P(ctypes.c_ssize_t), c_int, P(c_int)]),
    "MPI_Type_create_indexed_block": (c_int, [c_int, c_int, P(c_int), c_int, P(c_int)]),
    "MPI_Type_create_hindexed_block": (c_int, [c_int, c_int, P(ctypes.c_ssize_t), c_int, P(c_int)]),
    "MPI_Type_create_struct": (c_int, [c_int, P(c_int), P(ctypes.c_ssize_t), P(c_int), P(c_int)]),
    "MPI_Type_create_subarray": (c_int, [c_int, P(c_int), P(c_int), P(c_int), c_int, c_int, P(c_int)]),
    "MPI_Type_create_resized": (c_int, [c_int, ctypes.c_ssize_t, ctypes.c_ssize_t, P(c_int)]),
    "MPI_Type_dup": (c_int, [c_int, P(c_int)]),
    "MPI_Type_commit": (c_int, [P(c_int)]),
    "MPI_Type_free": (c_int, [P(c_int)]),
    "MPI_Type_size": (c_int, [c_int, P(c_int)]),
    "MPI_Type_get_extent": (c_int, [c_int, P(ctypes.c_ssize_t), P(ctypes.c_ssize_t)]),
    "MPI_Type_get_true_extent": (c_int, [c_int, P(ctypes.c_ssize_t), P(ctypes.c_ssize_t)]),
    "MPI_Pack": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int, P(c_int), c_int]),
    "MPI_Unpack": (c_int, [c_void_p, c_int, P(c_int), c_void_p, c_int, c_int, c_int]),
    "MPI_Pack_size": (c_int, [c_int, c_int, c_int, P(c_int)]),
    "MPI_Send": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int]),
    "MPI_Recv": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, P(Status)]),
    "MPI_Isend": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, P(c_int)]),
    "MPI_Irecv": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, P(c_int)]),
    "MPI_Wait": (c_int, [P(c_int), P(Status)]),
    "MPI_Get_count": (c_int, [P(Status), c_int, P(c_int)]),
    "MPI_Dist_graph_create_adjacent": (c_int, [c_int, c_int, c_void_p, c_void_p, c_int, c_void_p,
                                               c_void_p, c_int, c_int, P(c_int)]),
    "MPI_Dist_graph_neighbors_count": (c_int, [c_int, P(c_int), P(c_int), P(c_int)]),
    "MPI_Comm_free": (c_int, [P(c_int)]),
    "MPI_Neighbor_alltoallv": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                                       c_void_p, c_int, c_int]),
    "MPI_Neighbor_alltoallw": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                       c_void_p, c_void_p, c_void_p, c_int]),
    "MPI_Alltoallv": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                              c_void_p, c_int, c_int]),
    "MPI_Barrier": (c_int, [c_int]),
}

# the interposed entry points libtempi_b200.so must export
INTERPOSED = [
    "MPI_Init", "MPI_Init_thread", "MPI_Finalize", "MPI_Type_commit",
    "MPI_Type_free", "MPI_Pack", "MPI_Unpack", "MPI_Send", "MPI_Recv",
    "MPI_Isend", "MPI_Irecv", "MPI_Wait", "MPI_Neighbor_alltoallw", "MPI_Alltoallv",
]

_TEMPI_SIGS = {
    "tempi_pack": (c_int, [P(Desc), c_void_p, c_int64, c_void_p, P(Config), c_void_p]),
    "tempi_unpack": (c_int, [P(Desc), c_void_p, c_int64, c_void_p, P(Config), c_void_p]),
    "tempi_describe": (c_int, [c_int64, P(Desc)]),
    "tempi_batch_create": (c_int, [P(Region), ctypes.c_int32, ctypes.c_int32, P(c_void_p)]),
    "tempi_batch_launch": (c_int, [c_void_p, c_void_p]),
    "tempi_batch_capture": (c_int, [c_void_p, c_void_p]),
    "tempi_batch_replay": (c_int, [c_void_p, c_void_p]),
    "tempi_batch_destroy": (c_int, [c_void_p]),
    "tempi_batch_run_static": (c_int, [P(Region), ctypes.c_int32, ctypes.c_int32, c_void_p]),
    "tempi_batch_create_copy": (c_int, [P(CopyRegion), ctypes.c_int32, P(c_void_p)]),
    "tempi_batch_tune": (c_int, [c_void_p, c_void_p, ctypes.c_int32]),
    "tempi_batch_config": (c_int, [c_void_p, P(ctypes.c_int32), P(ctypes.c_int32),
                                   P(ctypes.c_int32), P(ctypes.c_int32), ctypes.c_int32]),
    "tempi_last_error": (ctypes.c_char_p, []),
    "tempi_kernel_launches": (c_int64, []),
    "tempi_last_kernel": (ctypes.c_char_p, []),
    "tempi_counter": (c_int64, [ctypes.c_char_p]),
    "tempi_staged_check": (c_int, []),
    "tempi_stream": (c_void_p, []),
    "tempi_features": (c_int, [P(Desc), c_int64, c_int, c_int, c_void_p]),
    "tempi_measure": (c_int, [P(Desc), c_int64, c_int, c_int, c_int, c_int, c_void_p]),
    "tempi_dispatch_load": (c_int, [ctypes.c_char_p, ctypes.c_char_p]),
    "tempi_dispatch_choose": (c_int, [P(Desc), c_int64, c_int, c_int, c_int, P(c_int),
                                      P(c_int), P(c_int), c_void_p, c_void_p]),
    "tempi_table_interp": (ctypes.c_double, [c_void_p, c_int, c_int, c_int64, c_int64]),
    "tempi_mlp_init": (c_int, [c_void_p, c_int, ctypes.c_uint64]),
    "tempi_mlp_train": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_int, c_int,
                                c_int, ctypes.c_float, ctypes.c_uint64, c_void_p, c_void_p]),
    "tempi_mlp_predict": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p]),
    "tempi_mlp_grad": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p,
                               c_void_p, c_void_p]),
    "tempi_reload_env": (c_int, []),
}


def counter(name: str) -> int:
    return tempi().tempi_counter(name.encode())


def _declare(lib, sigs, required=True):
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name, None) if not required else getattr(lib, name)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args


def minimpi():
    """The underlying (self-only) MPI library."""
    global _minimpi
    if _minimpi is None:
        tempi()
    return _minimpi


def _load_minimpi():
    global _minimpi
    if _minimpi is None:
        if not os.path.exists(MINIMPI_SO):
            raise ImportError(
                f"{MINIMPI_SO} is missing: build it with `make -C tempi_b200/csrc`"
            )
        _minimpi = ctypes.CDLL(MINIMPI_SO, mode=ctypes.RTLD_GLOBAL)
        _declare(_minimpi, _MPI_SIGS)
    return _minimpi


def tempi():
    """libtempi_b200.so: the interposed MPI entry points and the kernel ABI."""
    global _tempi
    if _tempi is None:
        if not os.path.exists(TEMPI_SO):
            raise ImportError(
                f"{TEMPI_SO} is missing: build it with `make -C tempi_b200/csrc`"
            )
        lib = ctypes.CDLL(TEMPI_SO, mode=ctypes.RTLD_GLOBAL)
        _declare(lib, {k: v for k, v in _MPI_SIGS.items() if k in INTERPOSED})
        _declare(lib, _TEMPI_SIGS, required=False)
        _load_minimpi()
        _tempi = lib
    return _tempi


def last_error() -> str:
    return tempi().tempi_last_error().decode(errors="replace")


def check(code: int, what: str = "tempi call") -> None:
    if code != 0:
        raise RuntimeError(f"{what} failed with code {code}: {last_error()}")
