"""ORACLE -- test infrastructure only.

ctypes front end of ``oracle/typemap.c`` (the C type-map walker).  Used by the
tests as the large-size checker and by ``bench.py`` as the timed CPU
baseline.  ``build()`` compiles it with gcc into ``oracle/liboracle.so``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from . import types as T

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

NODE_DTYPE = np.dtype(
    [
        ("kind", "<i4"),
        ("dense", "<i4"),
        ("child", "<i8"),
        ("count", "<i8"),
        ("bl", "<i8"),
        ("stride", "<i8"),
        ("size", "<i8"),
        ("lb", "<i8"),
        ("extent", "<i8"),
        ("aux", "<i8"),
    ]
)

_lib = None


def build() -> str:
    src = os.path.join(HERE, "typemap.c")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(
            ["gcc", "-O3", "-fPIC", "-shared", "-pthread", "-o", LIB, src]
        )
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
        _lib.oracle_walk.restype = ctypes.c_int64
        _lib.oracle_walk.argtypes = [
            ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
            ctypes.c_int, ctypes.c_int,
        ]
    return _lib


class Walker:
    """A lowered type, ready for repeated packs."""

    def __init__(self, t: T.OType):
        L, root = T.lower(t)
        self.t = t
        self.root = root
        self.nodes = np.zeros(len(L.nodes), NODE_DTYPE)
        for i, r in enumerate(L.nodes):
            self.nodes[i] = tuple(r)
        self.bls = np.asarray(L.bls + [0], np.int64)
        self.displs = np.asarray(L.displs + [0], np.int64)
        self.kids = np.asarray(L.kids + [0], np.int64)

    def _call(self, typed_ptr, incount, packed_ptr, unpack, nthreads):
        return lib().oracle_walk(
            self.nodes.ctypes.data, self.root, self.bls.ctypes.data,
            self.displs.ctypes.data, self.kids.ctypes.data, typed_ptr, incount,
            packed_ptr, unpack, nthreads,
        )

    def pack_into(self, buf: np.ndarray, incount: int, out: np.ndarray,
                  origin: int = 0, nthreads: int = 1) -> int:
        assert buf.dtype == np.uint8 and out.dtype == np.uint8
        assert out.nbytes >= incount * self.t.size
        return self._call(buf.ctypes.data + origin, incount, out.ctypes.data, 0,
                          nthreads)

    def pack(self, buf: np.ndarray, incount: int, origin: int = 0,
             nthreads: int = 1) -> np.ndarray:
        out = np.empty(incount * self.t.size, np.uint8)
        self.pack_into(buf, incount, out, origin, nthreads)
        return out

    def unpack(self, packed: np.ndarray, buf: np.ndarray, incount: int,
               origin: int = 0, nthreads: int = 1) -> int:
        assert buf.dtype == np.uint8 and packed.dtype == np.uint8
        return self._call(buf.ctypes.data + origin, incount, packed.ctypes.data,
                          1, nthreads)
