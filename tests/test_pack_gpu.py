"""Parity of the CUDA pack/unpack path with the oracle, through the C ABI.

Every check is byte-for-byte.  Unpack destinations are pre-filled with 0xAA
so that a write to a gap byte shows up as a mismatch (the reference's own
test pre-fills with the source pattern, test/pack_unpack.cpp:54-57, which
cannot see such writes).
"""
import ctypes

import numpy as np
import pytest

from oracle import types as T
from oracle import walker as W
from tempi_b200 import _lib, mpi

from . import helpers as H

pytestmark = pytest.mark.gpu


def dev(a: np.ndarray):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t) -> np.ndarray:
    return t.cpu().numpy()


def sync():
    import torch

    torch.cuda.synchronize()


def pack_dev(ty, src_np, count, origin=0):
    """MPI_Pack through the interposer with device buffers."""
    src = dev(src_np)
    out = dev(np.zeros(max(ty.o.size * count, 1), np.uint8))
    sync()
    err, pos = mpi.Pack(src.data_ptr() + origin, count, ty.h, out.data_ptr(), out.numel())
    assert err == 0, _lib.last_error()
    assert pos == ty.o.size * count
    return host(out)[: pos], src, out


def unpack_dev(ty, packed_dev, nbytes, count, origin=0):
    dst = dev(np.full(nbytes, 0xAA, np.uint8))
    sync()
    err, pos = mpi.Unpack(packed_dev.data_ptr(), ty.o.size * count, dst.data_ptr() + origin,
                          count, ty.h)
    assert err == 0, _lib.last_error()
    return host(dst)


def check_roundtrip(ty, count, seed=0, pattern=False):
    o = ty.o
    lo, hi = H.span(o, count)
    lo = min(lo, 0)
    nbytes = hi - lo + 64
    src = (np.arange(nbytes) & 0xFF).astype(np.uint8) if pattern else H.splitmix_bytes(nbytes, seed)
    want = W.Walker(o).pack(src, count, origin=-lo, nthreads=8)
    got, _, out = pack_dev(ty, src, count, origin=-lo)
    assert got.tobytes() == want.tobytes(), f"pack mismatch {ty.name} x{count}"
    exp = np.full(nbytes, 0xAA, np.uint8)
    W.Walker(o).unpack(want, exp, count, origin=-lo, nthreads=8)
    dst = unpack_dev(ty, out, nbytes, count, origin=-lo)
    assert dst.tobytes() == exp.tobytes(), f"unpack mismatch {ty.name} x{count}"


@pytest.mark.parametrize("case", range(13))
def test_reference_shapes(cuda, mpi_init, case):
    """Every shape of the reference's test/pack_unpack.cpp, src[i] = (char)i."""
    ty, count = H.reference_pack_cases()[case]
    ty.commit()
    check_roundtrip(ty, count, pattern=True)


def test_vector_1024x64_device(cuda, mpi_init):
    ty = H.make_2d_byte_vector(1024, 64, 512).commit()
    check_roundtrip(ty, 1, seed=0)
    assert _lib.counter("packs") > 0


def test_random_types(cuda, mpi_init):
    rng = np.random.default_rng(77)
    done = 0
    for _ in range(150):
        ty = H.random_type(rng).commit()
        if mpi.describe(ty.h)[0] != 0:
            continue
        check_roundtrip(ty, int(rng.integers(1, 4)), seed=int(rng.integers(0, 1 << 30)))
        done += 1
    assert done > 100


def test_golden_fixtures(cuda, mpi_init):
    import json
    import os

    gdir = os.path.join(os.path.dirname(__file__), "golden")
    for f in sorted(x for x in os.listdir(gdir) if x.endswith(".json")):
        g = json.load(open(os.path.join(gdir, f)))
        ty = _build_ty(g["type"]).commit()
        buf = H.splitmix_bytes(g["buf_bytes"], g["seed"])
        got, _, _ = pack_dev(ty, buf, g["incount"], origin=g["origin"])
        assert got.tobytes().hex() == g["packed_hex"], f


def _build_ty(spec):
    k = spec["kind"]
    if k == "named":
        return H.named({1: "BYTE", 4: "FLOAT", 8: "DOUBLE"}[spec["size"]])
    c = _build_ty(spec["child"])
    if k == "vector":
        return H.vector(spec["count"], spec["bl"], spec["stride"], c)
    if k == "hvector":
        return H.hvector(spec["count"], spec["bl"], spec["stride"], c)
    if k == "contiguous":
        return H.contiguous(spec["count"], c)
    if k == "subarray":
        return H.subarray(spec["sizes"], spec["subsizes"], spec["starts"], spec["order"], c)
    if k == "resized":
        return H.resized(c, spec["lb"], spec["extent"])
    raise ValueError(k)


def test_truncation_writes_nothing(cuda, mpi_init):
    ty = H.make_2d_byte_vector(64, 16, 32).commit()
    src = dev(H.splitmix_bytes(2048, 3))
    out = dev(np.full(512, 0x55, np.uint8))
    sync()
    err, pos = mpi.Pack(src.data_ptr(), 1, ty.h, out.data_ptr(), 512)
    assert err == mpi.ERR_TRUNCATE and pos == 0
    assert (host(out) == 0x55).all()
    err, pos = mpi.Unpack(out.data_ptr(), 100, src.data_ptr(), 1, ty.h)
    assert err == mpi.ERR_TRUNCATE


def test_positions_accumulate(cuda, mpi_init):
    """Several packs into one buffer at increasing positions, then unpacks."""
    a = H.make_2d_byte_vector(8, 5, 9).commit()
    b = H.subarray([6, 10], [3, 4], [2, 5], mpi.ORDER_C, H.named("FLOAT")).commit()
    sa, sb = H.splitmix_bytes(a.o.extent * 3, 1), H.splitmix_bytes(b.o.extent * 2, 2)
    da, db = dev(sa), dev(sb)
    total = a.o.size * 3 + b.o.size * 2
    out = dev(np.zeros(total, np.uint8))
    sync()
    err, pos = mpi.Pack(da.data_ptr(), 3, a.h, out.data_ptr(), total, 0)
    assert err == 0
    err, pos = mpi.Pack(db.data_ptr(), 2, b.h, out.data_ptr(), total, pos)
    assert err == 0 and pos == total
    want = np.concatenate([T.pack(a.o, sa, 3), T.pack(b.o, sb, 2)])
    assert host(out).tobytes() == want.tobytes()


def test_pack_into_pinned_host(cuda, mpi_init):
    """Mapped pinned host memory is device-accessible, so the kernel writes
    it directly (the ONE_SHOT store path)."""
    import torch

    ty = H.make_byte_v_hv((12, 7, 5), (40, 20, 10)).commit()
    src_np = H.splitmix_bytes(ty.o.extent * 2, 4)
    src = dev(src_np)
    out = torch.zeros(ty.o.size * 2, dtype=torch.uint8).pin_memory()
    sync()
    err, pos = mpi.Pack(src.data_ptr(), 2, ty.h, out.data_ptr(), out.numel())
    assert err == 0
    assert out.numpy().tobytes() == T.pack(ty.o, src_np, 2).tobytes()


@pytest.mark.parametrize("path", ["dma", "kernel"])
@pytest.mark.parametrize("shape", ["rows", "contiguous"])
def test_host_to_host_contiguous_run(cuda, mpi_init, path, shape):
    """Pinned host typed and packed buffers with objects that form one
    contiguous run (whole rows of a subarray at a start offset; three
    adjacent contiguous objects): the copy-engine pipeline (TEMPI_HOST_LINK
    unset) and the kernels (TEMPI_HOST_LINK=kernel) write the same bytes as
    the oracle, at an odd packed position, and the unpack leaves every byte
    outside the run alone."""
    import os

    import torch

    if shape == "rows":  # one object: rows 17..3016 of 4096, 12,288,000 B
        ty = H.subarray([4096, 1024], [3000, 1024], [17, 0], mpi.ORDER_C,
                        H.named("FLOAT")).commit()
        count = 1
    else:  # three adjacent objects of 1,000,003 floats
        ty = H.contiguous(1000003, H.named("FLOAT")).commit()
        count = 3
    assert ty.o.size * count >= 8 << 20
    old = os.environ.get("TEMPI_HOST_LINK")
    if path == "kernel":
        os.environ["TEMPI_HOST_LINK"] = "kernel"
    else:
        os.environ.pop("TEMPI_HOST_LINK", None)
    _lib.tempi().tempi_reload_env()
    try:
        src_np = H.splitmix_bytes(ty.o.extent * count, 21)
        src = torch.from_numpy(src_np).pin_memory()
        pos0 = 5
        packed = torch.zeros(ty.o.size * count + pos0 + 3, dtype=torch.uint8).pin_memory()
        n0 = _lib.counter("host_link_copies")
        err, pos = mpi.Pack(src.data_ptr(), count, ty.h, packed.data_ptr(), packed.numel(), pos0)
        assert err == 0 and pos == pos0 + ty.o.size * count
        want = T.pack(ty.o, src_np, count)
        assert packed.numpy()[pos0:pos].tobytes() == want.tobytes()
        assert not packed.numpy()[:pos0].any() and not packed.numpy()[pos:].any()
        back = torch.full_like(src, 0xAA).pin_memory()
        err, upos = mpi.Unpack(packed.data_ptr(), packed.numel(), back.data_ptr(), count, ty.h, pos0)
        assert err == 0 and upos == pos
        exp = np.full_like(src_np, 0xAA)
        T.unpack(ty.o, want, exp, count)
        assert back.numpy().tobytes() == exp.tobytes()
        used = _lib.counter("host_link_copies") - n0
        assert used == (2 if path == "dma" else 0)
    finally:
        if old is None:
            os.environ.pop("TEMPI_HOST_LINK", None)
        else:
            os.environ["TEMPI_HOST_LINK"] = old
        _lib.tempi().tempi_reload_env()


def test_host_link_small_chunks(cuda, mpi_init):
    """The copy-engine pipeline with TEMPI_HOST_LINK_CHUNK_KB=256: a contiguous
    run of 9 MiB + 12 B between pinned host buffers goes through 37 chunks,
    each of the 4 staging slots reused 9 times, with a short last chunk; the
    pack and the unpack write the oracle's bytes and nothing else."""
    import os

    import torch

    ty = H.contiguous((9 << 20) // 4 + 3, H.named("FLOAT")).commit()
    os.environ["TEMPI_HOST_LINK_CHUNK_KB"] = "256"
    _lib.tempi().tempi_reload_env()
    try:
        src_np = H.splitmix_bytes(ty.o.extent, 41)
        src = torch.from_numpy(src_np).pin_memory()
        packed = torch.zeros(ty.o.size + 16, dtype=torch.uint8).pin_memory()
        n0 = _lib.counter("host_link_copies")
        err, pos = mpi.Pack(src.data_ptr(), 1, ty.h, packed.data_ptr(), packed.numel(), 16)
        assert err == 0 and pos == 16 + ty.o.size
        assert packed.numpy()[16:].tobytes() == src_np.tobytes()
        assert not packed.numpy()[:16].any()
        back = torch.full_like(src, 0xAA).pin_memory()
        err, upos = mpi.Unpack(packed.data_ptr(), packed.numel(), back.data_ptr(), 1, ty.h, 16)
        assert err == 0 and upos == pos
        assert back.numpy().tobytes() == src_np.tobytes()
        assert _lib.counter("host_link_copies") - n0 == 2
    finally:
        del os.environ["TEMPI_HOST_LINK_CHUNK_KB"]
        _lib.tempi().tempi_reload_env()


@pytest.mark.parametrize("path", ["dma", "kernel"])
@pytest.mark.parametrize("shape", ["rows256_odd", "rows1000", "rows64_odd", "two_dims"])
def test_host_to_host_strided_rows(cuda, mpi_init, path, shape):
    """Pinned host typed and packed buffers with objects whose bytes are rows
    of one strided dimension: the unpack by the copy-engine 2-D path (rows of
    128 B or more, TEMPI_HOST_LINK unset) or by the kernels writes only the
    rows, and the pack (kernels) writes the oracle's bytes at an odd packed
    position.  Rows of 64 B, and a layout with two strided dimensions, stay
    on the kernels either way."""
    import os

    import torch

    if shape == "rows256_odd":  # 3-D subarray of floats, 256-B rows at byte 28
        ty = H.subarray([256, 256, 256], [256, 256, 64], [0, 0, 7], mpi.ORDER_C,
                        H.named("FLOAT")).commit()
        count, rows = 1, True
    elif shape == "rows1000":  # 1000-B rows at 1040 B, 3 objects continuing the rows
        ty = H.resized(H.hvector(3000, 1000, 1040, H.named("BYTE")), 0, 3000 * 1040).commit()
        count, rows = 3, True
    elif shape == "rows64_odd":  # 64-B rows at byte 120: below the 2-D path's row width
        ty = H.subarray([256, 256, 256], [256, 256, 16], [0, 0, 30], mpi.ORDER_C,
                        H.named("FLOAT")).commit()
        count, rows = 2, False
    else:  # a column block of a 2-D subarray repeated with a gap: two dimensions
        ty = H.resized(H.subarray([2048, 2048], [2000, 512], [3, 7], mpi.ORDER_C,
                                  H.named("FLOAT")), 0, 2048 * 2048 * 4 + 4096).commit()
        count, rows = 3, False
    assert ty.o.size * count >= 8 << 20
    old = os.environ.get("TEMPI_HOST_LINK")
    if path == "kernel":
        os.environ["TEMPI_HOST_LINK"] = "kernel"
    else:
        os.environ.pop("TEMPI_HOST_LINK", None)
    _lib.tempi().tempi_reload_env()
    try:
        src_np = H.splitmix_bytes(ty.o.extent * count + 64, 23)
        src = torch.from_numpy(src_np).pin_memory()
        pos0 = 7
        packed = torch.zeros(ty.o.size * count + pos0 + 5, dtype=torch.uint8).pin_memory()
        n0 = _lib.counter("host_link_copies")
        err, pos = mpi.Pack(src.data_ptr(), count, ty.h, packed.data_ptr(), packed.numel(), pos0)
        assert err == 0 and pos == pos0 + ty.o.size * count
        want = T.pack(ty.o, src_np, count)
        assert packed.numpy()[pos0:pos].tobytes() == want.tobytes()
        assert not packed.numpy()[:pos0].any() and not packed.numpy()[pos:].any()
        back = torch.full_like(src, 0xAA).pin_memory()
        err, upos = mpi.Unpack(packed.data_ptr(), packed.numel(), back.data_ptr(), count, ty.h, pos0)
        assert err == 0 and upos == pos
        exp = np.full_like(src_np, 0xAA)
        T.unpack(ty.o, want, exp, count)
        assert back.numpy().tobytes() == exp.tobytes()
        used = _lib.counter("host_link_copies") - n0
        assert used == (1 if path == "dma" and rows else 0)
    finally:
        if old is None:
            os.environ.pop("TEMPI_HOST_LINK", None)
        else:
            os.environ["TEMPI_HOST_LINK"] = old
        _lib.tempi().tempi_reload_env()


@pytest.mark.parametrize("where", ["host_host", "host_dev", "dev_host"])
def test_every_configuration_on_host_memory(cuda, mpi_init, where):
    """Every kernel configuration the dispatcher can pick (word kernel at 3
    block sizes, row kernel, shift kernel at 4/8/16/32 lanes) reading or
    writing pinned host memory over the link, on layouts with misaligned
    wide rows, short rows and a packed position that is not 16-B aligned:
    the bytes match the oracle both ways and the unpack leaves gaps alone."""
    import torch

    from tests.test_canon import desc_pack

    configs = [(1, 256, 0), (1, 512, 0), (1, 128, 0), (2, 256, 0),
               (3, 256, 4), (3, 256, 8), (3, 256, 16), (3, 256, 32)]
    cases = [
        _lib.Desc.make(540, 256 * 1024, 256, [96], [1024]),           # 256-B rows at +12
        _lib.Desc.make(244, 40000, 1000, [3, 5], [1300, 4 * 1300]),   # 1000-B rows, 2 dims
        _lib.Desc.make(120, 64 * 1024, 64, [200], [320]),             # 64-B rows over lines
        _lib.Desc.make(3, 9000, 20, [7, 11], [36, 7 * 40]),           # short odd rows
    ]
    pmis = 7
    for d in cases:
        incount = 2
        span = d.start + d.extent * (incount - 1) + d.block + 64
        for k in range(d.ndims):
            span += d.strides[k] * (d.counts[k] - 1)
        src_np = H.splitmix_bytes(span, d.block)
        want = desc_pack(d, src_np, incount)
        typed_host = where in ("host_host", "host_dev")
        packed_host = where in ("host_host", "dev_host")

        def buf(a, on_host):
            t = torch.from_numpy(np.ascontiguousarray(a))
            return t.pin_memory() if on_host else t.cuda()

        src = buf(src_np, typed_host)
        for kernel, threads, lanes in configs:
            cfg = _lib.Config(kernel, 0, threads, lanes, 0, 0)
            out = buf(np.zeros(d.size * incount + pmis + 9, np.uint8), packed_host)
            sync()
            _lib.check(_lib.tempi().tempi_pack(ctypes.byref(d), src.data_ptr(), incount,
                                                out.data_ptr() + pmis, ctypes.byref(cfg), None))
            sync()
            got = out.cpu().numpy()
            assert got[pmis:pmis + d.size * incount].tobytes() == want.tobytes(), (d.block, kernel, lanes)
            back = buf(np.full_like(src_np, 0xAA), typed_host)
            sync()
            _lib.check(_lib.tempi().tempi_unpack(ctypes.byref(d), out.data_ptr() + pmis, incount,
                                                  back.data_ptr(), ctypes.byref(cfg), None))
            sync()
            exp = np.full_like(src_np, 0xAA)
            shape = [incount] + [d.counts[k] for k in reversed(range(d.ndims))] + [d.block]
            strides = [d.extent] + [d.strides[k] for k in reversed(range(d.ndims))] + [1]
            v = np.lib.stride_tricks.as_strided(exp[d.start:], shape=shape, strides=strides,
                                                writeable=True)
            v[...] = want.reshape(v.shape)
            assert back.cpu().numpy().tobytes() == exp.tobytes(), (d.block, kernel, lanes)


@pytest.mark.parametrize("kernel", [1, 2])
@pytest.mark.parametrize("width", [1, 2, 4, 8, 16])
@pytest.mark.parametrize("threads", [64, 256, 512])
def test_kernel_variants(cuda, mpi_init, kernel, width, threads):
    """Every kernel variant, width and block size writes the same bytes."""
    import torch

    cases = [
        _lib.Desc.make(48, 1 << 20, 256, [100, 7], [1024, 1024 * 128]),
        _lib.Desc.make(16, 112 * 4096, 64, [4096], [64 + 16 * 3]),
        _lib.Desc.make(0, 8192 * 33, 4096, [33], [4096 * 2]),
        _lib.Desc.make(32, 1 << 16, 32, [3, 5, 7, 2], [64, 256, 2048, 20000]),
    ]
    for d in cases:
        incount = 3
        o_span = d.start + d.extent * (incount - 1) + 1
        for k in range(d.ndims):
            o_span += d.strides[k] * (d.counts[k] - 1)
        o_span += d.block + 64
        src_np = H.splitmix_bytes(o_span, 9)
        src = dev(src_np)
        out = torch.zeros(d.size * incount, dtype=torch.uint8, device="cuda")
        cfg = _lib.Config(kernel, width, threads, 0, 0, 0)
        _lib.check(_lib.tempi().tempi_pack(ctypes.byref(d), src.data_ptr(), incount,
                                            out.data_ptr(), ctypes.byref(cfg), None))
        sync()
        from tests.test_canon import desc_pack

        want = desc_pack(d, src_np, incount)
        assert host(out).tobytes() == want.tobytes()
        back = torch.full_like(src, 0xAA)
        _lib.check(_lib.tempi().tempi_unpack(ctypes.byref(d), out.data_ptr(), incount,
                                              back.data_ptr(), ctypes.byref(cfg), None))
        sync()
        b = host(back)
        exp = np.full_like(src_np, 0xAA)
        v = np.lib.stride_tricks.as_strided(
            exp[d.start:], shape=[incount] + [d.counts[k] for k in reversed(range(d.ndims))] + [d.block],
            strides=[d.extent] + [d.strides[k] for k in reversed(range(d.ndims))] + [1], writeable=True)
        v[...] = want.reshape(v.shape)
        assert b.tobytes() == exp.tobytes()


@pytest.mark.parametrize("lanes", [4, 8, 16, 32])
def test_shift_kernel_every_misalignment(cuda, mpi_init, lanes):
    """The funnel-shift row kernel (kernel 3) at every source and packed
    misalignment 0..15 and row lengths around the 16-B word boundaries."""
    import torch

    from tests.test_canon import desc_pack

    for block in (1, 15, 16, 17, 31, 33, 100, 255, 256, 257, 1000, 2100):
        for mis in (0, 1, 2, 3, 4, 5, 7, 8, 9, 12, 13, 15):
            d = _lib.Desc.make(mis, 64 * 1024, block, [9, 3], [block + 37, 9 * (block + 37) + 3])
            incount = 2
            src_np = H.splitmix_bytes(d.extent * incount + 64, block * 16 + mis)
            src = dev(src_np)
            pmis = (mis * 7) % 16  # also misalign the packed side
            out = torch.zeros(d.size * incount + 32, dtype=torch.uint8, device="cuda")
            cfg = _lib.Config(3, 0, 128, lanes, 0, 0)
            _lib.check(_lib.tempi().tempi_pack(ctypes.byref(d), src.data_ptr(), incount,
                                                out.data_ptr() + pmis, ctypes.byref(cfg), None))
            sync()
            want = desc_pack(d, src_np, incount)
            got = host(out)[pmis: pmis + d.size * incount]
            assert got.tobytes() == want.tobytes(), (block, mis, lanes)
            back = torch.full_like(src, 0xAA)
            _lib.check(_lib.tempi().tempi_unpack(ctypes.byref(d), out.data_ptr() + pmis, incount,
                                                  back.data_ptr(), ctypes.byref(cfg), None))
            sync()
            exp = np.full_like(src_np, 0xAA)
            v = np.lib.stride_tricks.as_strided(
                exp[d.start:], shape=[incount, 3, 9, block],
                strides=[d.extent, d.strides[1], d.strides[0], 1], writeable=True)
            v[...] = want.reshape(v.shape)
            assert host(back).tobytes() == exp.tobytes(), (block, mis, lanes)
            assert _lib.tempi().tempi_last_kernel().decode() == f"shift_unpack_l{lanes}"


SWEEP_2D = [(c, 1024) for c in (1, 2, 4, 8, 16, 64, 256, 1024)]
SWEEP_3D = [(c, 256, 256) for c in (1, 2, 4, 8, 16, 64, 256)]


@pytest.mark.parametrize("inner,rows", SWEEP_2D)
@pytest.mark.parametrize("incount", [1, 16])
def test_sweep_2d_full_size(cuda, mpi_init, inner, rows, incount):
    """The strided sweep, 2-D: float subarrays of a 1024x1024 array at full
    size, starts from a seed, compared with the oracle's C walker."""
    rng = np.random.default_rng(inner * 31 + incount)
    sc = int(rng.integers(0, 1024 - inner + 1))
    ty = H.subarray([1024, 1024], [rows, inner], [0, sc], mpi.ORDER_C, H.named("FLOAT")).commit()
    check_roundtrip(ty, incount, seed=inner)


@pytest.mark.parametrize("inner,mid,outer", SWEEP_3D)
def test_sweep_3d_full_size(cuda, mpi_init, inner, mid, outer):
    rng = np.random.default_rng(inner)
    s0 = int(rng.integers(0, 256 - inner + 1))
    ty = H.subarray([256, 256, 256], [outer, mid, inner], [0, 0, s0], mpi.ORDER_C,
                    H.named("FLOAT")).commit()
    check_roundtrip(ty, 4 if inner >= 64 else 1, seed=inner + 100)


def test_sweep_equivalent_constructors(cuda, mpi_init):
    """The same pattern as a subarray, an hvector of vectors and a
    contiguous of hvectors packs identically (the sweep's variants)."""
    C, r, c, sr, sc = 1024, 96, 24, 5, 13
    sub = H.subarray([1024, C], [r, c], [sr, sc], mpi.ORDER_C, H.named("FLOAT")).commit()
    hv = H.resized(H.hvector(r, 1, 4 * C, H.vector(1, c, c, H.named("FLOAT"))), 0, 4 * C * 1024).commit()
    ch = H.contiguous(1, H.hvector(r, c, 4 * C, H.named("FLOAT"))).commit()
    src = H.splitmix_bytes(4 * C * 1024 + 64, 5)
    origin = 4 * (sc + sr * C)
    a, _, _ = pack_dev(sub, src, 1)
    b, _, _ = pack_dev(hv, src, 1, origin=origin)
    c_, _, _ = pack_dev(ch, src, 1, origin=origin)
    assert a.tobytes() == b.tobytes() == c_.tobytes() == T.pack(sub.o, src, 1).tobytes()


def _cudart():
    import ctypes as C
    import os as _os

    import nvidia.cuda_runtime as cr

    rt = C.CDLL(_os.path.join(list(cr.__path__)[0], "lib", "libcudart.so.12"))
    rt.cudaMallocManaged.argtypes = [C.POINTER(C.c_void_p), C.c_size_t, C.c_uint]
    rt.cudaFree.argtypes = [C.c_void_p]
    rt.cudaDeviceSynchronize.argtypes = []
    return rt


@pytest.mark.parametrize("case", range(13))
def test_reference_shapes_on_managed_memory(cuda, mpi_init, case):
    """The reference's pack test allocates its buffers with cudaMallocManaged
    (test/pack_unpack.cpp): the same shapes on managed memory go through the
    interposer's GPU path, bit-exact both ways, gaps untouched."""
    rt = _cudart()
    ty, count = H.reference_pack_cases()[case]
    ty.commit()
    o = ty.o
    lo, hi = H.span(o, count)
    lo = min(lo, 0)
    nbytes = hi - lo + 64
    ptrs = []

    def managed(n):
        p = ctypes.c_void_p()
        assert rt.cudaMallocManaged(ctypes.byref(p), max(n, 1), 1) == 0  # attach global
        ptrs.append(p.value)
        return p.value, np.ctypeslib.as_array((ctypes.c_uint8 * max(n, 1)).from_address(p.value))

    try:
        sp, src = managed(nbytes)
        src[:] = (np.arange(nbytes) & 0xFF).astype(np.uint8)  # src[i] = (char)i
        pp, packed = managed(o.size * count)
        up, dst = managed(nbytes)
        dst[:] = 0xAA
        assert rt.cudaDeviceSynchronize() == 0
        n0 = _lib.counter("packs")
        err, pos = mpi.Pack(sp - lo, count, ty.h, pp, o.size * count)
        assert err == 0 and pos == o.size * count, _lib.last_error()
        assert _lib.counter("packs") == n0 + 1  # the GPU path, not the library
        err, _ = mpi.Unpack(pp, o.size * count, up - lo, count, ty.h)
        assert err == 0, _lib.last_error()
        assert rt.cudaDeviceSynchronize() == 0
        want = W.Walker(o).pack(src.copy(), count, origin=-lo)
        assert packed[:pos].tobytes() == want.tobytes()
        exp = np.full(nbytes, 0xAA, np.uint8)
        W.Walker(o).unpack(want, exp, count, origin=-lo)
        assert dst.tobytes() == exp.tobytes()
    finally:
        for p in ptrs:
            rt.cudaFree(p)


def test_offsets_beyond_4gib(cuda, mpi_init):
    """Rows more than 4 GiB from the origin (the reference's >4 GiB case is
    compiled out, test/pack_unpack.cpp:139-155): three 100-byte rows 2 GiB +
    13 bytes apart, as one object and as two objects 3 GiB apart."""
    import torch

    step = (2 << 30) + 13
    d = _lib.Desc.make(7, 3 * step, 100, [3], [step])
    total = 7 + 2 * step + 100 + 256
    buf = torch.zeros(total, dtype=torch.uint8, device="cuda")
    rows = [H.splitmix_bytes(100, 60 + i) for i in range(3)]
    for i, r in enumerate(rows):
        buf[7 + i * step: 7 + i * step + 100] = torch.from_numpy(r).cuda()
    out = torch.zeros(300, dtype=torch.uint8, device="cuda")
    _lib.check(_lib.tempi().tempi_pack(ctypes.byref(d), buf.data_ptr(), 1, out.data_ptr(),
                                        None, None))
    torch.cuda.synchronize()
    assert out.cpu().numpy().tobytes() == np.concatenate(rows).tobytes()
    # unpack into the same places after clearing them; the bytes around stay 0
    for i in range(3):
        buf[7 + i * step: 7 + i * step + 100] = 0
    _lib.check(_lib.tempi().tempi_unpack(ctypes.byref(d), out.data_ptr(), 1, buf.data_ptr(),
                                          None, None))
    torch.cuda.synchronize()
    for i, r in enumerate(rows):
        at = 7 + i * step
        got = buf[at - 7: at + 107].cpu().numpy()
        assert got[7:107].tobytes() == r.tobytes()
        assert not got[:7].any() and not got[107:].any()
    del buf
    torch.cuda.empty_cache()
    # two objects, the second at 3 GiB: rows at 3 GiB + 5 and 3 GiB + 5 + 1 GiB
    d2 = _lib.Desc.make(5, 3 << 30, 64, [2], [1 << 30])
    total = 5 + (3 << 30) + (1 << 30) + 64 + 64
    buf = torch.zeros(total, dtype=torch.uint8, device="cuda")
    offs = [5, 5 + (1 << 30), 5 + (3 << 30), 5 + (3 << 30) + (1 << 30)]
    rows = [H.splitmix_bytes(64, 70 + i) for i in range(4)]
    for o, r in zip(offs, rows):
        buf[o: o + 64] = torch.from_numpy(r).cuda()
    out = torch.zeros(256, dtype=torch.uint8, device="cuda")
    _lib.check(_lib.tempi().tempi_pack(ctypes.byref(d2), buf.data_ptr(), 2, out.data_ptr(),
                                        None, None))
    torch.cuda.synchronize()
    assert out.cpu().numpy().tobytes() == np.concatenate(rows).tobytes()
    del buf
    torch.cuda.empty_cache()


def test_staged_unpack_matches_oracle(cuda, mpi_init):
    """The staged unpack (kernel 4: packed chunks pulled into shared memory
    by bulk copies, then scattered) at every typed-side width, with one to
    three strided dimensions, several objects, sizes that leave a partial
    last chunk, and a packed side that is not 16-B aligned (where it must
    hand over to the plain kernels).  Gap bytes keep their 0xAA fill and no
    bounded wait gives up."""
    import torch

    from tests.test_canon import desc_pack

    cases = [  # (desc, incount): typed-side widths 4, 8, 1, 2, 16
        (_lib.Desc.make(540, 1 << 20, 256, [1000], [1024]), 2),
        (_lib.Desc.make(120, 300 * 1024, 64, [17, 300], [1024, 17 * 1024]), 1),
        (_lib.Desc.make(3, 70000, 48, [1200], [57]), 1),
        (_lib.Desc.make(2, 14000, 32, [5, 7, 9], [34, 200, 1500]), 3),
        # 16-B aligned rows of 512 B and more, and a contiguous run: the bulk
        # kernel (bulk stores per row piece; partial last chunks)
        (_lib.Desc.make(0, 1 << 20, 4096, [60], [8192]), 2),
        (_lib.Desc.make(16, 200 * 2080 + 64, 528, [13, 15], [1040, 13 * 1040 + 48]), 3),
        (_lib.Desc.make(32, (3 << 20) + 1296, (3 << 20) + 1264, [], []), 2),
    ]
    before = _lib.counter("staged_timeouts")
    for d, incount in cases:
        span = d.start + d.extent * (incount - 1) + d.block + 64
        for k in range(d.ndims):
            span += d.strides[k] * (d.counts[k] - 1)
        src_np = H.splitmix_bytes(span, d.block + incount)
        want = desc_pack(d, src_np, incount)
        assert want.size % 16 == 0
        exp = np.full_like(src_np, 0xAA)
        shape = [incount] + [d.counts[k] for k in reversed(range(d.ndims))] + [d.block]
        strides = [d.extent] + [d.strides[k] for k in reversed(range(d.ndims))] + [1]
        np.lib.stride_tricks.as_strided(exp[d.start:], shape=shape, strides=strides,
                                        writeable=True)[...] = want.reshape(shape)
        for mis in (0, 4):  # 4: the packed base is not 16-B aligned
            packed = torch.zeros(want.size + 32, dtype=torch.uint8, device="cuda")
            packed[mis: mis + want.size] = torch.from_numpy(want).cuda()
            dst = torch.full((span,), 0xAA, dtype=torch.uint8, device="cuda")
            cfg = _lib.Config(4, 0, 256, 0, 0, 0)
            _lib.check(_lib.tempi().tempi_unpack(ctypes.byref(d), packed.data_ptr() + mis,
                                                  incount, dst.data_ptr(), ctypes.byref(cfg),
                                                  None))
            sync()
            kname = _lib.tempi().tempi_last_kernel().decode()
            assert kname.startswith("staged") == (mis == 0), (kname, d.block)
            assert host(dst).tobytes() == exp.tobytes(), (d.block, incount, mis)
    assert _lib.counter("staged_timeouts") == before == 0


def test_staged_pack_matches_oracle(cuda, mpi_init):
    """The staged pack (kernel 4 on the pack side: row pieces gathered into
    shared memory by bulk copies, written out by bulk stores) on
    16-B aligned geometries: rows of 16 B (hundreds of pieces per chunk),
    rows that chunks cut in the middle, a contiguous run with a partial last
    chunk, and enough chunks that each CTA cycles its stages several times
    (one CTA per SM).  A geometry narrower than 16 B hands over to the plain
    kernels.  Bytes past the packed size stay untouched and no bounded wait
    gives up."""
    import torch

    from tests.test_canon import desc_pack

    cases = [  # (desc, incount, staged)
        (_lib.Desc.make(0, 1 << 20, 4096, [60], [8192]), 2, True),
        (_lib.Desc.make(32, 64 * 1040 + 64, 400, [64], [1040]), 3, True),
        (_lib.Desc.make(16, 1 << 20, 16, [7, 9, 5], [48, 1024, 16384]), 4, True),
        (_lib.Desc.make(0, (8 << 20) + 48, (8 << 20) + 48, [], []), 1, True),
        (_lib.Desc.make(4, 1 << 20, 4096, [60], [8192]), 1, False),
    ]
    before = _lib.counter("staged_timeouts")
    for d, incount, staged in cases:
        span = d.start + d.extent * (incount - 1) + d.block + 64
        for k in range(d.ndims):
            span += d.strides[k] * (d.counts[k] - 1)
        src_np = H.splitmix_bytes(span, d.block + incount + 5)
        want = desc_pack(d, src_np, incount)
        src = torch.from_numpy(src_np).cuda()
        for bps in (1, 8):
            packed = torch.full((want.size + 256,), 0x5A, dtype=torch.uint8, device="cuda")
            cfg = _lib.Config(4, 0, 256, 0, bps, 0)
            _lib.check(_lib.tempi().tempi_pack(ctypes.byref(d), src.data_ptr(), incount,
                                                packed.data_ptr(), ctypes.byref(cfg), None))
            sync()
            kname = _lib.tempi().tempi_last_kernel().decode()
            assert kname.startswith("staged") == staged, (kname, d.block)
            got = host(packed)
            assert got[:want.size].tobytes() == want.tobytes(), (d.block, incount, bps)
            assert (got[want.size:] == 0x5A).all(), (d.block, incount, bps)
    assert _lib.counter("staged_timeouts") == before == 0
    assert _lib.tempi().tempi_staged_check() == 0


@pytest.mark.parametrize("kernel", [1, 2, 3])
def test_plain_kernels_random_geometries(cuda, mpi_init, kernel):
    """The word, row and shift kernels, forced, on 60 seeded random
    non-overlapping descriptors (zero to four strided dimensions, one to five
    objects, every alignment of block, start and packed offset, 128 to 512
    threads, 4 to 32 lanes per row for the shift kernel): each pack equals the
    descriptor oracle and each unpack writes exactly the described bytes."""
    import torch

    from tests.test_canon import desc_pack

    rng = np.random.default_rng(900 + kernel)
    lib = _lib.tempi()
    for case in range(60):
        nd = int(rng.integers(0, 5))
        unit = int(rng.choice([1, 2, 4, 8, 16]))
        block = unit * int(rng.integers(1, 120 if nd else 4000))
        counts, strides, span = [], [], block
        for k in range(nd):
            c = int(rng.integers(2, 30))
            st = span + int(rng.integers(0, 40))  # any alignment, past everything inside
            counts.append(c)
            strides.append(st)
            span = st * (c - 1) + span
        incount = int(rng.integers(1, 6))
        extent = span + int(rng.integers(0, 24))
        start = int(rng.integers(0, 24))
        d = _lib.Desc.make(start, extent, block, counts, strides)
        total = d.size * incount
        if total == 0 or total > (1 << 20):
            continue
        nbytes = start + extent * (incount - 1) + span + 64
        src_np = H.splitmix_bytes(nbytes, 3000 + case)
        want = desc_pack(d, src_np, incount)
        src = torch.from_numpy(src_np).cuda()
        poff = int(rng.integers(0, 17))
        threads = int(rng.choice([128, 256, 512])) if kernel != 3 else 256
        lanes = int(rng.choice([4, 8, 16, 32])) if kernel == 3 else 0
        cfg = _lib.Config(kernel, 0, threads, lanes, 0, 0)
        packed = torch.full((total + poff + 64,), 0x5A, dtype=torch.uint8, device="cuda")
        _lib.check(lib.tempi_pack(ctypes.byref(d), src.data_ptr(), incount,
                                  packed.data_ptr() + poff, ctypes.byref(cfg), None))
        sync()
        got = host(packed)
        assert got[poff:poff + total].tobytes() == want.tobytes(), (case, d.as_dict(), incount)
        assert (got[:poff] == 0x5A).all() and (got[poff + total:] == 0x5A).all(), case
        dst = torch.full((nbytes,), 0xAA, dtype=torch.uint8, device="cuda")
        _lib.check(lib.tempi_unpack(ctypes.byref(d), packed.data_ptr() + poff, incount,
                                    dst.data_ptr(), ctypes.byref(cfg), None))
        sync()
        exp = np.full(nbytes, 0xAA, np.uint8)
        shape = [incount] + [d.counts[k] for k in reversed(range(d.ndims))] + [d.block]
        strd = [d.extent] + [d.strides[k] for k in reversed(range(d.ndims))] + [1]
        np.lib.stride_tricks.as_strided(exp[d.start:], shape=shape, strides=strd,
                                        writeable=True)[...] = want.reshape(shape)
        assert host(dst).tobytes() == exp.tobytes(), (case, d.as_dict(), incount)


def test_staged_random_geometries(cuda, mpi_init):
    """The staged kernels (kernel 4) on 100 seeded random descriptors: zero to
    four strided dimensions that do not overlap, one to five objects, block
    lengths with and without the 16-B alignment the staged pack needs, start
    offsets and packed offsets at every alignment (the kernels take what they
    can and hand the rest to the plain kernels), and 1, 3 or 8 CTAs per SM.
    Each pack equals the descriptor oracle and each unpack writes exactly the
    described bytes; no bounded wait gives up."""
    import torch

    from tests.test_canon import desc_pack

    rng = np.random.default_rng(4711)
    lib = _lib.tempi()
    staged_runs = 0
    for case in range(100):
        nd = int(rng.integers(0, 5))
        aligned = bool(rng.integers(0, 2))
        unit = 16 if aligned else int(rng.choice([1, 2, 4, 8]))
        block = unit * int(rng.integers(1, 200 if nd else 40000))
        counts, strides, span = [], [], block
        for k in range(nd):
            c = int(rng.integers(2, 40))
            st = span + unit * int(rng.integers(0, 8))  # past everything inside
            counts.append(c)
            strides.append(st)
            span = st * (c - 1) + span
        incount = int(rng.integers(1, 6))
        extent = span + unit * int(rng.integers(0, 4))
        start = unit * int(rng.integers(0, 4))
        d = _lib.Desc.make(start, extent, block, counts, strides)
        total = d.size * incount
        if total == 0 or total > (3 << 20):
            continue
        nbytes = start + extent * (incount - 1) + span + 64
        src_np = H.splitmix_bytes(nbytes, 1000 + case)
        want = desc_pack(d, src_np, incount)
        src = torch.from_numpy(src_np).cuda()
        poff = int(rng.choice([0, 16, 4])) if not aligned else 0
        bps = int(rng.choice([1, 3, 8]))
        cfg = _lib.Config(4, 0, 256, 0, bps, 0)
        packed = torch.full((total + poff + 64,), 0x5A, dtype=torch.uint8, device="cuda")
        _lib.check(lib.tempi_pack(ctypes.byref(d), src.data_ptr(), incount,
                                  packed.data_ptr() + poff, ctypes.byref(cfg), None))
        sync()
        staged_runs += lib.tempi_last_kernel().decode().startswith("staged")
        got = host(packed)
        assert got[poff:poff + total].tobytes() == want.tobytes(), (case, d.as_dict(), incount)
        assert (got[:poff] == 0x5A).all() and (got[poff + total:] == 0x5A).all(), case
        dst = torch.full((nbytes,), 0xAA, dtype=torch.uint8, device="cuda")
        _lib.check(lib.tempi_unpack(ctypes.byref(d), packed.data_ptr() + poff, incount,
                                    dst.data_ptr(), ctypes.byref(cfg), None))
        sync()
        staged_runs += lib.tempi_last_kernel().decode().startswith("staged")
        exp = np.full(nbytes, 0xAA, np.uint8)
        shape = [incount] + [d.counts[k] for k in reversed(range(d.ndims))] + [d.block]
        strd = [d.extent] + [d.strides[k] for k in reversed(range(d.ndims))] + [1]
        np.lib.stride_tricks.as_strided(exp[d.start:], shape=shape, strides=strd,
                                        writeable=True)[...] = want.reshape(shape)
        assert host(dst).tobytes() == exp.tobytes(), (case, d.as_dict(), incount)
    assert staged_runs >= 30
    assert lib.tempi_staged_check() == 0


def test_staged_give_up_is_reported(cuda, mpi_init):
    """A staged kernel whose bounded waits run out must not pass for a good
    copy.  TEMPI_TEST_STAGED_SHORTFALL makes every chunk's barrier expect 16
    bytes more than its bulk copy delivers, so each wait gives up after about
    a second: tempi_staged_check then reports TEMPI_ERR_TIMEOUT (once), the
    counter moves, and the interposed MPI_Unpack returns an error instead of
    MPI_SUCCESS.  With the knob cleared the same calls copy correctly again
    on the same context."""
    import os

    import torch

    from tests.test_canon import desc_pack

    lib = _lib.tempi()
    # 1 MiB packed, rows of 256 B: 128 chunks, one per CTA, so each CTA
    # waits once and has no other copies to drain
    d = _lib.Desc.make(0, 1 << 22, 256, [4096], [1024])
    span = d.block + d.strides[0] * (d.counts[0] - 1)
    src_np = H.splitmix_bytes(span, 77)
    want = desc_pack(d, src_np, 1)
    packed = torch.from_numpy(want).cuda()
    exp = np.full(span, 0xAA, np.uint8)
    T.unpack(T.hvector(4096, 256, 1024, T.BYTE), want, exp, 1)
    cfg = _lib.Config(4, 0, 256, 0, 8, 0)
    t = mpi.Type_create_hvector(4096, 256, 1024, mpi.BYTE)
    assert mpi.Type_commit(t) == 0
    before = _lib.counter("staged_timeouts")
    assert lib.tempi_staged_check() == 0
    os.environ["TEMPI_TEST_STAGED_SHORTFALL"] = "16"
    os.environ["TEMPI_DISPATCH"] = "heuristic"  # fixed rules: staged for this unpack
    try:
        lib.tempi_reload_env()
        dst = torch.full((span,), 0xAA, dtype=torch.uint8, device="cuda")
        _lib.check(lib.tempi_unpack(ctypes.byref(d), packed.data_ptr(), 1, dst.data_ptr(),
                                    ctypes.byref(cfg), None))
        sync()
        assert lib.tempi_last_kernel().decode().startswith("staged")
        assert lib.tempi_staged_check() == 4  # TEMPI_ERR_TIMEOUT
        assert lib.tempi_staged_check() == 0  # reported once
        assert _lib.counter("staged_timeouts") == before + 1
        err, _ = mpi.Unpack(packed.data_ptr(), want.size, dst.data_ptr(), 1, t)
        assert err != 0
        assert lib.tempi_last_kernel().decode().startswith("staged")
        assert _lib.counter("staged_timeouts") == before + 2
    finally:
        del os.environ["TEMPI_TEST_STAGED_SHORTFALL"]
        del os.environ["TEMPI_DISPATCH"]
        lib.tempi_reload_env()
    dst = torch.full((span,), 0xAA, dtype=torch.uint8, device="cuda")
    _lib.check(lib.tempi_unpack(ctypes.byref(d), packed.data_ptr(), 1, dst.data_ptr(),
                                ctypes.byref(cfg), None))
    sync()
    assert lib.tempi_staged_check() == 0
    assert host(dst).tobytes() == exp.tobytes()
    err, _ = mpi.Unpack(packed.data_ptr(), want.size, dst.data_ptr(), 1, t)
    assert err == 0 and host(dst).tobytes() == exp.tobytes()
    assert _lib.counter("staged_timeouts") == before + 2
    mpi.Type_free(t)


@pytest.mark.parametrize("unpack", [0, 1])
def test_bulk_give_up_is_reported(cuda, mpi_init, unpack):
    """The bulk kernels (the staged pack, and the staged unpack of wide
    aligned rows) under TEMPI_TEST_STAGED_SHORTFALL: every chunk's barrier
    expects 16 bytes more than its copies bring, so each bounded wait gives
    up; the launch reports TEMPI_ERR_TIMEOUT once, and the same call on the
    same context is exact once the knob is cleared."""
    import os

    import torch

    from tests.test_canon import desc_pack

    lib = _lib.tempi()
    # 1 MiB packed in rows of 1 KiB, 16-B aligned: 64 chunks of 16 KB, one
    # per CTA, so each CTA waits once and drains one chunk
    d = _lib.Desc.make(0, 1 << 21, 1024, [1024], [2048])
    span = d.block + d.strides[0] * (d.counts[0] - 1)
    src_np = H.splitmix_bytes(span, 91)
    want = desc_pack(d, src_np, 1)
    exp = np.full(span, 0xAA, np.uint8)
    T.unpack(T.hvector(1024, 1024, 2048, T.BYTE), want, exp, 1)
    cfg = _lib.Config(4, 0, 256, 0, 3, 0)
    src = torch.from_numpy(src_np).cuda()
    packed = torch.from_numpy(want).cuda()

    def run():
        if unpack:
            out = torch.full((span,), 0xAA, dtype=torch.uint8, device="cuda")
            _lib.check(lib.tempi_unpack(ctypes.byref(d), packed.data_ptr(), 1, out.data_ptr(),
                                        ctypes.byref(cfg), None))
        else:
            out = torch.zeros(want.size, dtype=torch.uint8, device="cuda")
            _lib.check(lib.tempi_pack(ctypes.byref(d), src.data_ptr(), 1, out.data_ptr(),
                                      ctypes.byref(cfg), None))
        sync()
        assert lib.tempi_last_kernel().decode().startswith("staged")
        return host(out)

    before = _lib.counter("staged_timeouts")
    assert lib.tempi_staged_check() == 0
    os.environ["TEMPI_TEST_STAGED_SHORTFALL"] = "16"
    try:
        lib.tempi_reload_env()
        run()
        assert lib.tempi_staged_check() == 4  # TEMPI_ERR_TIMEOUT
        assert lib.tempi_staged_check() == 0  # reported once
        assert _lib.counter("staged_timeouts") == before + 1
    finally:
        del os.environ["TEMPI_TEST_STAGED_SHORTFALL"]
        lib.tempi_reload_env()
    got = run()
    assert lib.tempi_staged_check() == 0
    assert got.tobytes() == (exp if unpack else want).tobytes()
