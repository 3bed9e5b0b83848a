"""The product canonicaliser (tempi_describe, run at MPI_Type_commit), on CPU.

A descriptor is correct when walking it -- block bytes at
start + sum i_k * strides[k], fastest dim first, object j at j*extent --
visits exactly the bytes MPI type-map order visits.  That is checked here
with a numpy strided view against the oracle, for the reference's factories
(support/type.cpp) and for random nested types.
"""
import numpy as np
import pytest

from oracle import refcanon as R
from oracle import types as T
from tempi_b200 import mpi

from . import helpers as H


def desc_pack(d, buf, incount, origin=0):
    """Pack by walking a tempi_desc (numpy restatement of the kernel's job)."""
    n = d.ndims
    shape = [incount] + [d.counts[k] for k in reversed(range(n))] + [d.block]
    strides = [d.extent] + [d.strides[k] for k in reversed(range(n))] + [1]
    base = origin + d.start
    # as_strided wants a base view; negative strides are fine from `base`
    v = np.lib.stride_tricks.as_strided(buf[base:], shape=shape, strides=strides)
    return np.ascontiguousarray(v).ravel()


def test_vector_1024x64_descriptor(mpi_init):
    t = H.make_2d_byte_vector(1024, 64, 512).commit()
    err, d = mpi.describe(t.h)
    assert err == 0
    assert d.as_dict() == dict(start=0, extent=523840, block=64, size=65536, ndims=1,
                               align=16, counts=[1024], strides=[512])


def test_matches_reference_strided_block_when_reference_is_right(mpi_init):
    """Where the reference's canonicaliser keeps MPI order, TEMPI's
    descriptor is the same strided block (counts[0] of the reference is the
    block length here)."""
    for ty, _ in H.reference_pack_cases():
        ty.commit()
        err, d = mpi.describe(ty.h)
        assert err == 0
        sb = R.canonicalize(ty.o)
        if sb.ndims == 0:
            continue
        assert d.start == sb.start and d.block == sb.counts[0]
        assert [d.counts[k] for k in range(d.ndims)] == sb.counts[1:]
        assert [d.strides[k] for k in range(d.ndims)] == sb.strides[1:]


def test_hv_by_cols_keeps_mpi_order(mpi_init):
    t = H.make_2d_hv_by_cols(13, 3, 16, 5, 53).commit()
    err, d = mpi.describe(t.h)
    assert err == 0
    assert (d.block, d.ndims, d.counts[0], d.strides[0], d.counts[1], d.strides[1]) == (13, 2, 5, 53, 3, 16)
    buf = H.splitmix_bytes(600, 1)
    assert desc_pack(d, buf, 1).tobytes() == T.pack(t.o, buf, 1).tobytes()


@pytest.mark.parametrize("factory", ["v1", "vn", "sub", "contig"])
def test_contiguous_factories_are_one_block(mpi_init, factory):
    f = {"v1": H.make_contiguous_byte_v1, "vn": H.make_contiguous_byte_vn,
         "sub": H.make_contiguous_subarray, "contig": H.make_contiguous_contiguous}[factory]
    for n in (1, 2, 3, 4, 100):
        t = f(n).commit()
        err, d = mpi.describe(t.h)
        assert err == 0 and d.ndims == 0 and d.block == n and d.extent == n


def test_3d_equivalence_class_same_descriptor(mpi_init):
    ae, ce = (256, 512, 1024), (100, 13, 47)
    ts = [H.make_byte_v_hv(ce, ae), H.make_byte_v1_hv_hv(ce, ae),
          H.make_byte_vn_hv_hv(ce, ae), H.make_hib(ce, ae), H.make_hi(ce, ae)]
    descs = []
    for t in ts:
        t.commit()
        err, d = mpi.describe(t.h)
        descs.append((err, d.start, d.block, tuple(d.counts[: d.ndims]), tuple(d.strides[: d.ndims])))
    # hindexed(_block) over two levels is not regular: those go to the library
    assert descs[0] == descs[1] == descs[2] == (0, 0, 100, (13, 47), (256, 256 * 512))
    assert descs[3][0] == 3 and descs[4][0] == 3


def test_unsupported_types(mpi_init):
    st = H.struct([1, 1], [0, 8], [H.named("INT"), H.named("DOUBLE")]).commit()
    assert mpi.describe(st.h)[0] == 3
    irregular = H.hindexed([2, 3], [0, 10], H.named()).commit()
    assert mpi.describe(irregular.h)[0] == 3
    regular = H.hindexed([3, 3, 3], [0, 10, 20], H.named()).commit()
    err, d = mpi.describe(regular.h)
    assert err == 0 and d.block == 3 and d.counts[0] == 3 and d.strides[0] == 10


def test_random_types_descriptor_walk_matches_typemap(mpi_init):
    rng = np.random.default_rng(2024)
    checked = 0
    for _ in range(400):
        ty = H.random_type(rng).commit()
        err, d = mpi.describe(ty.h)
        if err == 3:
            continue
        assert err == 0
        o = ty.o
        assert d.size == o.size and d.extent == o.extent
        for cnt in (1, 3):
            lo, hi = H.span(o, cnt)
            lo = min(lo, 0)
            buf = H.splitmix_bytes(hi - lo + 32, int(rng.integers(0, 1 << 30)))
            want = T.pack(o, buf, cnt, origin=-lo)
            got = desc_pack(d, buf, cnt, origin=-lo)
            assert got.tobytes() == want.tobytes(), ty.name
        checked += 1
    assert checked > 300


def test_fortran_subarray_descriptor(mpi_init):
    t = H.subarray([7, 9, 5], [3, 4, 2], [1, 2, 3], mpi.ORDER_FORTRAN, H.named("FLOAT")).commit()
    err, d = mpi.describe(t.h)
    assert err == 0
    buf = H.splitmix_bytes(t.o.extent * 3, 9)
    assert desc_pack(d, buf, 3).tobytes() == T.pack(t.o, buf, 3).tobytes()


def test_alignment_proof(mpi_init):
    t = H.subarray([64, 64], [8, 16], [3, 5], mpi.ORDER_C, H.named("FLOAT")).commit()
    err, d = mpi.describe(t.h)
    assert err == 0 and d.block == 64 and d.align == 4  # start 4*(5+3*64) is 4-aligned
    t2 = H.subarray([64, 64], [8, 16], [3, 4], mpi.ORDER_C, H.named("FLOAT")).commit()
    assert mpi.describe(t2.h)[1].align == 16
