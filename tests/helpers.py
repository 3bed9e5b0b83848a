"""Shared test helpers.

``Ty`` pairs an MPI datatype handle (built through the underlying MPI
library) with the oracle's independent description of the same type, so a
test can pack through TEMPI and check against the oracle.  The factories
mirror the reference's support/type.cpp:3-310 one for one.
"""
from __future__ import annotations

import numpy as np

from oracle import types as T
from tempi_b200 import mpi


class Ty:
    def __init__(self, h: int, o: T.OType, name: str = ""):
        self.h = h
        self.o = o
        self.name = name

    def commit(self):
        assert mpi.Type_commit(self.h) == 0
        return self

    def __repr__(self):
        return f"Ty({self.name})"


NAMED = {
    "BYTE": (mpi.BYTE, T.BYTE),
    "FLOAT": (mpi.FLOAT, T.FLOAT),
    "DOUBLE": (mpi.DOUBLE, T.DOUBLE),
    "INT": (mpi.INT, T.INT),
}


def named(n="BYTE"):
    h, o = NAMED[n]
    return Ty(h, o, n)


def contiguous(count, c: Ty):
    return Ty(mpi.Type_contiguous(count, c.h), T.contiguous(count, c.o),
              f"contig({count},{c.name})")


def vector(count, bl, stride, c: Ty):
    return Ty(mpi.Type_vector(count, bl, stride, c.h), T.vector(count, bl, stride, c.o),
              f"vector({count},{bl},{stride},{c.name})")


def hvector(count, bl, stride, c: Ty):
    return Ty(mpi.Type_create_hvector(count, bl, stride, c.h),
              T.hvector(count, bl, stride, c.o), f"hvector({count},{bl},{stride},{c.name})")


def subarray(sizes, subsizes, starts, order, c: Ty):
    oo = T.ORDER_C if order == mpi.ORDER_C else T.ORDER_FORTRAN
    return Ty(mpi.Type_create_subarray(sizes, subsizes, starts, order, c.h),
              T.subarray(sizes, subsizes, starts, oo, c.o),
              f"subarray({sizes},{subsizes},{starts},{'C' if order == mpi.ORDER_C else 'F'},{c.name})")


def hindexed(bls, displs, c: Ty):
    return Ty(mpi.Type_create_hindexed(bls, displs, c.h), T.hindexed(bls, displs, c.o),
              f"hindexed({bls},{displs},{c.name})")


def hindexed_block(bl, displs, c: Ty):
    return Ty(mpi.Type_create_hindexed_block(bl, displs, c.h),
              T.hindexed_block(bl, displs, c.o), f"hib({bl},{c.name})")


def indexed_block(bl, displs, c: Ty):
    return Ty(mpi.Type_create_indexed_block(bl, displs, c.h),
              T.indexed_block(bl, displs, c.o), f"ib({bl},{c.name})")


def resized(c: Ty, lb, extent):
    return Ty(mpi.Type_create_resized(c.h, lb, extent), T.resized(c.o, lb, extent),
              f"resized({c.name},{lb},{extent})")


def dup(c: Ty):
    return Ty(mpi.Type_dup(c.h), T.dup(c.o), f"dup({c.name})")


def struct(bls, displs, tys):
    return Ty(mpi.Type_create_struct(bls, displs, [t.h for t in tys]),
              T.struct(bls, displs, [t.o for t in tys]), "struct")


# ---- the reference's support/type.cpp factories (x = fastest) ---------------


def make_byte_vn_hv_hv(ce, ae):
    row = vector(ce[0], 1, 1, named())
    plane = hvector(ce[1], 1, ae[0], row)
    return hvector(ce[2], 1, ae[0] * ae[1], plane)


def make_byte_v1_hv_hv(ce, ae):
    row = vector(1, ce[0], ae[0], named())
    plane = hvector(ce[1], 1, ae[0], row)
    return hvector(ce[2], 1, ae[0] * ae[1], plane)


def make_byte_v_hv(ce, ae):
    plane = vector(ce[1], ce[0], ae[0], named())
    return hvector(ce[2], 1, ae[0] * ae[1], plane)


def make_float_v_hv(ce, ae):
    plane = vector(ce[1], ce[0] // 4, ae[0] // 4, named("FLOAT"))
    return hvector(ce[2], 1, ae[0] * ae[1], plane)


def make_hi(ce, ae):
    displs = [z * ae[1] * ae[0] + y * ae[0] for z in range(ce[2]) for y in range(ce[1])]
    return hindexed([ce[0]] * len(displs), displs, named())


def make_hib(ce, ae):
    displs = [z * ae[1] * ae[0] + y * ae[0] for z in range(ce[2]) for y in range(ce[1])]
    return hindexed_block(ce[0], displs, named())


def make_subarray(ce, ae):
    return subarray([ae[2], ae[1], ae[0]], [ce[2], ce[1], ce[0]], [0, 0, 0], mpi.ORDER_C,
                    named())


def make_subarray_v(ce, ae):
    plane = subarray([ae[1], ae[0]], [ce[1], ce[0]], [0, 0], mpi.ORDER_C, named())
    return vector(ce[2], 1, 1, plane)


def make_off_subarray(ce, ae, off):
    # note: this factory lists dims in (x, y, z) order as the outermost first,
    # exactly like support/type.cpp:199-211
    return subarray([ae[0], ae[1], ae[2]], [ce[0], ce[1], ce[2]], [off[0], off[1], off[2]],
                    mpi.ORDER_C, named())


def make_2d_byte_vector(nb, bl, st):
    return vector(nb, bl, st, named())


def make_2d_byte_hvector(nb, bl, st):
    return hvector(nb, bl, st, named())


def make_2d_byte_subarray(nb, bl, st):
    return subarray([nb, st], [nb, bl], [0, 0], mpi.ORDER_C, named())


def make_2d_hv_by_rows(bs, c1, s1, c2, s2):
    b = contiguous(bs, named())
    row = hvector(c1, 1, s1, b)
    return hvector(c2, 1, s2, row)


def make_2d_hv_by_cols(bs, c1, s1, c2, s2):
    b = contiguous(bs, named())
    col = hvector(c2, 1, s2, b)
    return hvector(c1, 1, s1, col)


def make_contiguous_byte_v1(n):
    return vector(n, 1, 1, named())


def make_contiguous_byte_vn(n):
    return vector(1, n, n, named())


def make_contiguous_subarray(n):
    return subarray([n], [n], [0], mpi.ORDER_C, named())


def make_contiguous_contiguous(n):
    return contiguous(n, named())


# (type, incount) cases of the reference's test/pack_unpack.cpp:157-302
def reference_pack_cases():
    cases = [(make_contiguous_contiguous(10), 30)]
    for count in (1, 2):
        cases.append((make_2d_byte_vector(2, 3, 4), count))
    for count in (1, 2):
        cases.append((make_2d_byte_subarray(2, 3, 4), count))
    cases.append((make_off_subarray((2, 3, 4), (16, 16, 16), (1, 1, 4)), 1))
    for count in (1, 2):
        cases.append((make_off_subarray((2, 3, 4), (16, 16, 16), (1, 1, 4)), count))
    cases.append((make_byte_v_hv((2, 3, 4), (10, 10, 10)), 1))
    cases.append((make_byte_v_hv((2, 3, 4), (10, 10, 10)), 2))
    cases.append((make_byte_v_hv((10, 10, 1), (10, 10, 10)), 1))
    cases.append((make_byte_v_hv((4, 3, 4), (200, 200, 200)), 1))
    cases.append((make_byte_v_hv((100, 100, 100), (200, 200, 200)), 1))
    cases.append((make_byte_v_hv((100, 100, 100), (200, 200, 200)), 3))
    return cases


# ---- seeded data --------------------------------------------------------------


def splitmix_bytes(n: int, seed: int) -> np.ndarray:
    """Seeded uniform bytes (numpy PCG64 from a fixed seed)."""
    return np.random.default_rng(seed).integers(0, 256, n, dtype=np.uint8)


def span(o: T.OType, incount: int):
    """(lo, hi) byte span, relative to the origin, of `incount` objects."""
    if incount == 0 or o.size == 0:
        return 0, 0
    a, b = 0, (incount - 1) * o.extent
    return min(a, b) + o.true_lb, max(a, b) + o.true_ub


def random_type(rng, max_bytes=1 << 16):
    """A random nesting of vector/hvector/subarray/contiguous/resized over a
    named type, kept below `max_bytes` of extent."""
    base = named(["BYTE", "FLOAT", "DOUBLE", "INT"][rng.integers(0, 4)])
    t = base
    depth = int(rng.integers(1, 4))
    for _ in range(depth):
        kind = int(rng.integers(0, 5))
        e = max(t.o.extent, 1)
        if kind == 0:
            cnt = int(rng.integers(1, 6))
            bl = int(rng.integers(1, 4))
            stride = bl + int(rng.integers(0, 4))
            cand = vector(cnt, bl, stride, t)
        elif kind == 1:
            cnt = int(rng.integers(1, 6))
            bl = int(rng.integers(1, 3))
            stride = bl * e + int(rng.integers(0, 17))
            cand = hvector(cnt, bl, stride, t)
        elif kind == 2:
            nd = int(rng.integers(1, 4))
            sizes = [int(rng.integers(1, 7)) for _ in range(nd)]
            subs = [int(rng.integers(1, s + 1)) for s in sizes]
            starts = [int(rng.integers(0, s - b + 1)) for s, b in zip(sizes, subs)]
            order = mpi.ORDER_C if rng.integers(0, 2) else mpi.ORDER_FORTRAN
            cand = subarray(sizes, subs, starts, order, t)
        elif kind == 3:
            cand = contiguous(int(rng.integers(1, 5)), t)
        else:
            cand = resized(t, 0, t.o.extent + int(rng.integers(0, 9)))
        if cand.o.extent > max_bytes or cand.o.size == 0:
            break
        t = cand
    return t
