"""Pins the oracle (CPU only).

The reference stores no golden files: its pack test compares TEMPI against
the system MPI_Pack at run time (test/pack_unpack.cpp:19-126).  The oracle is
pinned here by (1) the known answers the reference's tests do hold
(test/measure_system.cpp, test/type_equivalence.cpp, the worked examples of
src/internal/types.cpp), (2) agreement of three independent pack
implementations -- numpy type-map expansion, the C walker, and the
restatement of the reference canonicaliser + packers -- on every shape of
test/pack_unpack.cpp, and (3) the committed golden fixtures.
"""
import json
import os

import numpy as np
import pytest

from oracle import interp as I
from oracle import refcanon as R
from oracle import types as T
from oracle import walker as W

from . import helpers as H

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_interp_time_known_answers():
    # test/measure_system.cpp:13-38
    v = [2, 4, 8, 16]
    assert [I.interp_time(v, b) for b in (1, 2, 3, 5, 7)] == [2, 4, 6, 10, 14]


def test_interp_2d_known_answers():
    # test/measure_system.cpp:41-92
    a = [[14, 18, 22], [16, 20, 24]]
    cases = {(64, 1): 14, (160, 1): 15, (256, 1): 16, (64, 2): 18, (256, 2): 20,
             (64, 3): 20, (64, 4): 22, (160, 3): 21, (512, 1): 32, (512, 3): 44}
    for (b, s), want in cases.items():
        assert I.interp_2d(a, b, s) == want, (b, s)


def test_log2_known_answers():
    # include/numeric.hpp log2_floor/log2_ceil
    assert [I.log2_floor(x) for x in (0, 1, 2, 3, 4, 5, 1023, 1024)] == [0, 0, 1, 1, 2, 2, 9, 10]
    assert [I.log2_ceil(x) for x in (1, 2, 3, 4, 5, 1023, 1024, 1025)] == [0, 1, 2, 2, 3, 10, 10, 11]


def test_vector_1024x64_strided_block():
    # worked example: MPI_Type_vector(1024,64,512,MPI_BYTE)
    t = T.vector(1024, 64, 512, T.BYTE)
    assert (t.size, t.lb, t.extent) == (65536, 0, 523840)
    sb = R.canonicalize(t)
    assert (sb.start, sb.extent, sb.counts, sb.strides) == (0, 523840, [64, 1024], [1, 512])


def test_subarray_2d_float_block():
    # C-order 2-D float subarray -> counts [4c, r], strides [1, 4C], start 4(sc+sr*C)
    R_, C_, r, c, sr, sc = 64, 96, 5, 7, 3, 11
    sb = R.canonicalize(T.subarray([R_, C_], [r, c], [sr, sc], T.ORDER_C, T.FLOAT))
    assert sb.counts == [4 * c, r] and sb.strides == [1, 4 * C_]
    assert sb.start == 4 * (sc + sr * C_) and sb.extent == 4 * R_ * C_


def test_type_equivalence_known_answers():
    # test/type_equivalence.cpp:176-196
    rows = T.hvector(5, 1, 53, T.hvector(3, 1, 16, T.contiguous(13, T.BYTE)))
    cols = T.hvector(3, 1, 16, T.hvector(5, 1, 53, T.contiguous(13, T.BYTE)))
    for t in (rows, cols):
        assert t.size == 15 * 13
        assert t.extent == 53 * 4 + 16 * 2 + 13
    # :31-58 contiguous factories agree on size, lb, extent
    for n in (1, 2, 3, 4):
        ts = [T.vector(n, 1, 1, T.BYTE), T.vector(1, n, n, T.BYTE),
              T.subarray([n], [n], [0], T.ORDER_C, T.BYTE), T.contiguous(n, T.BYTE)]
        assert len({(t.size, t.lb, t.extent) for t in ts}) == 1


@pytest.mark.parametrize("case", range(13))
def test_three_oracles_agree_on_reference_shapes(mpi_init, case):
    """Every test/pack_unpack.cpp shape: numpy type map == C walker == the
    reference canonicaliser + packer restatement (that test's own check)."""
    ty, count = H.reference_pack_cases()[case]
    o = ty.o
    buf = (np.arange(o.extent * count + 64) & 0xFF).astype(np.uint8)  # src[i] = (char)i
    a = T.pack(o, buf, count)
    b = W.Walker(o).pack(buf, count)
    c = R.ref_pack(R.canonicalize(o), buf, count)
    assert a.tobytes() == b.tobytes() == c.tobytes()
    # unpack restores every described byte and only those
    dst = np.full_like(buf, 0xAA)
    W.Walker(o).unpack(a, dst, count)
    exp = np.full_like(buf, 0xAA)
    T.unpack(o, a, exp, count)
    assert dst.tobytes() == exp.tobytes()


def test_reference_canonicaliser_reorders_columns():
    """The reference's stream_swap (types.cpp:378-404) makes an hvector of
    columns pack in row order, which is not MPI's type-map order."""
    cols = T.hvector(3, 1, 16, T.hvector(5, 1, 53, T.contiguous(13, T.BYTE)))
    rows = T.hvector(5, 1, 53, T.hvector(3, 1, 16, T.contiguous(13, T.BYTE)))
    assert R.canonicalize(cols) == R.canonicalize(rows)
    buf = H.splitmix_bytes(600, 7)
    mpi_order = T.pack(cols, buf, 1)
    ref_order = R.ref_pack(R.canonicalize(cols), buf, 1)
    assert sorted(mpi_order.tolist()) == sorted(ref_order.tolist())
    assert mpi_order.tobytes() != ref_order.tobytes()


def test_hib_hi_vhv_pack_identically():
    # test/type_equivalence.cpp:60-171 intends this (its loop packs types[0]
    # every time); here the five constructors really are compared
    ae, ce = (32, 24, 8), (10, 13, 5)
    ts = [T.hindexed_block(ce[0], [z * ae[1] * ae[0] + y * ae[0] for z in range(ce[2]) for y in range(ce[1])], T.BYTE),
          T.hindexed([ce[0]] * ce[1] * ce[2], [z * ae[1] * ae[0] + y * ae[0] for z in range(ce[2]) for y in range(ce[1])], T.BYTE),
          T.hvector(ce[2], 1, ae[0] * ae[1], T.vector(ce[1], ce[0], ae[0], T.BYTE)),
          T.hvector(ce[2], 1, ae[0] * ae[1], T.hvector(ce[1], 1, ae[0], T.vector(1, ce[0], ae[0], T.BYTE))),
          T.hvector(ce[2], 1, ae[0] * ae[1], T.hvector(ce[1], 1, ae[0], T.vector(ce[0], 1, 1, T.BYTE)))]
    buf = H.splitmix_bytes(int(np.prod(ae)), 3)
    packs = {T.pack(t, buf, 1).tobytes() for t in ts}
    assert len(packs) == 1
    assert len({t.size for t in ts}) == 1


def test_c_walker_threads_match(mpi_init):
    o = T.vector(4096, 24, 40, T.BYTE)
    buf = H.splitmix_bytes(o.extent * 3, 11)
    w = W.Walker(o)
    one = w.pack(buf, 3, nthreads=1)
    many = w.pack(buf, 3, nthreads=8)
    single = w.pack(buf, 1, nthreads=8)
    assert one.tobytes() == many.tobytes()
    assert single.tobytes() == one[: o.size].tobytes()


def test_c_walker_thread_split_through_wrappers():
    """Threaded walks split a subarray (start displacement wrapper), a
    resized type and a count-1 vector wrapper at their inner vector's
    blocks; every split must write what one thread writes, for pack and
    unpack, with one object and with several."""
    sub = T.subarray([64, 48, 40], [30, 20, 16], [5, 7, 9], T.ORDER_C, T.named(4))
    res = T.resized(T.vector(37, 3, 5, T.named(2)), -8, 500)
    wrap = T.hvector(1, 1, 0, T.vector(50, 7, 9, T.BYTE))
    fort = T.subarray([33, 12], [20, 5], [3, 4], T.ORDER_FORTRAN, T.named(8))
    for o in (sub, res, wrap, fort):
        w = W.Walker(o)
        for cnt in (1, 3):
            lo = min(0, o.true_lb)
            hi = o.true_ub + (cnt - 1) * o.extent
            buf = H.splitmix_bytes(hi - lo + 16, cnt)
            one = w.pack(buf, cnt, origin=-lo, nthreads=1)
            assert one.tobytes() == T.pack(o, buf, cnt, origin=-lo).tobytes()
            for nt in (2, 7, 64):
                assert w.pack(buf, cnt, origin=-lo, nthreads=nt).tobytes() == one.tobytes()
                a = np.zeros_like(buf)
                b = np.zeros_like(buf)
                w.unpack(one, a, cnt, origin=-lo, nthreads=1)
                w.unpack(one, b, cnt, origin=-lo, nthreads=nt)
                assert a.tobytes() == b.tobytes()


def test_random_types_numpy_vs_c_walker():
    rng = np.random.default_rng(5)
    for _ in range(200):
        o = _random_otype(rng)
        cnt = int(rng.integers(1, 4))
        lo = min(0, o.true_lb + min(0, (cnt - 1) * o.extent))
        hi = max(o.true_ub + max(0, (cnt - 1) * o.extent), 1)
        buf = H.splitmix_bytes(hi - lo + 16, int(rng.integers(0, 1 << 30)))
        a = T.pack(o, buf, cnt, origin=-lo)
        b = W.Walker(o).pack(buf, cnt, origin=-lo)
        assert a.tobytes() == b.tobytes()


def _random_otype(rng):
    t = [T.BYTE, T.FLOAT, T.DOUBLE][rng.integers(0, 3)]
    for _ in range(int(rng.integers(1, 4))):
        k = int(rng.integers(0, 6))
        e = t.extent
        if k == 0:
            t = T.vector(int(rng.integers(1, 5)), int(rng.integers(1, 3)), int(rng.integers(-4, 6)), t)
        elif k == 1:
            t = T.hvector(int(rng.integers(1, 5)), int(rng.integers(1, 3)), int(rng.integers(-2 * e, 3 * e + 9)), t)
        elif k == 2:
            nd = int(rng.integers(1, 4))
            sizes = [int(rng.integers(1, 6)) for _ in range(nd)]
            subs = [int(rng.integers(1, s + 1)) for s in sizes]
            starts = [int(rng.integers(0, s - b + 1)) for s, b in zip(sizes, subs)]
            t = T.subarray(sizes, subs, starts, [T.ORDER_C, T.ORDER_FORTRAN][rng.integers(0, 2)], t)
        elif k == 3:
            t = T.contiguous(int(rng.integers(1, 4)), t)
        elif k == 4:
            t = T.resized(t, int(rng.integers(-3, 3)), e + int(rng.integers(0, 9)))
        else:
            n = int(rng.integers(1, 4))
            t = T.hindexed([int(rng.integers(1, 3)) for _ in range(n)],
                           [int(rng.integers(-20, 60)) for _ in range(n)], t)
        if t.extent > 4096 or t.size == 0:
            break
    return t


def test_golden_fixtures_match_oracle():
    """tests/golden/*.json hold the packed bytes of seeded cases, made by
    tests/golden/make_golden.py."""
    files = sorted(f for f in os.listdir(GOLDEN) if f.endswith(".json"))
    assert files, "no golden fixtures"
    for f in files:
        g = json.load(open(os.path.join(GOLDEN, f)))
        o = _build_otype(g["type"])
        buf = H.splitmix_bytes(g["buf_bytes"], g["seed"])
        packed = T.pack(o, buf, g["incount"], origin=g["origin"])
        assert packed.tobytes().hex() == g["packed_hex"], f
        assert W.Walker(o).pack(buf, g["incount"], origin=g["origin"]).tobytes().hex() == g["packed_hex"]


def _build_otype(spec):
    k = spec["kind"]
    if k == "named":
        return T.named(spec["size"])
    c = _build_otype(spec["child"])
    if k == "vector":
        return T.vector(spec["count"], spec["bl"], spec["stride"], c)
    if k == "hvector":
        return T.hvector(spec["count"], spec["bl"], spec["stride"], c)
    if k == "contiguous":
        return T.contiguous(spec["count"], c)
    if k == "subarray":
        return T.subarray(spec["sizes"], spec["subsizes"], spec["starts"], spec["order"], c)
    if k == "resized":
        return T.resized(c, spec["lb"], spec["extent"])
    raise ValueError(k)
