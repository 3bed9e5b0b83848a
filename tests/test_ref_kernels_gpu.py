"""The reference's own packer kernels (include/pack_kernels.cuh, compiled from
the reference sources into oracle/_ref by oracle/build_ref.sh) against this
library's kernels and the oracle, on the same B200.

Parity: on shapes where the reference is correct (its word size must divide
every stride and the base pointer, which it does not check), the reference
packers, TEMPI's kernels and the type-map oracle write the same bytes.

Timing: both kernels on the same buffers, CUDA events on one stream; the
table is printed, and written to $TEMPI_RESULTS_DIR/ref_vs_tempi.json when
that variable names a directory.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from oracle import refcanon as R
from oracle import types as T
from tempi_b200 import _lib, mpi

from . import helpers as H

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libref_pack.so")


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref/libref_pack.so was not built (reference sources absent)")
    lib = ctypes.CDLL(REF_SO)
    u, v = ctypes.c_uint, ctypes.c_void_p
    lib.ref_pack_2d.argtypes = [ctypes.c_int, v, v, ctypes.c_int, u, u, u, u, u, v]
    lib.ref_pack_3d.argtypes = [ctypes.c_int, v, v, ctypes.c_int, u, u, u, u, u, u, u, v]
    return lib


def ref_launch(ref, sb, unpack, typed, packed, incount, stream=None):
    if sb.ndims == 2:
        return ref.ref_pack_2d(unpack, typed, packed, incount, sb.start, sb.counts[0],
                               sb.counts[1], sb.strides[1], sb.extent, stream)
    assert sb.ndims == 3
    return ref.ref_pack_3d(unpack, typed, packed, incount, sb.start, sb.counts[0],
                           sb.counts[1], sb.strides[1], sb.counts[2], sb.strides[2],
                           sb.extent, stream)


def cases():
    """(name, Ty, incount) where the reference's word size divides every
    stride, so its kernels are correct."""
    out = [("vector_1024x64_s512", H.make_2d_byte_vector(1024, 64, 512), 1)]
    out.append(("2d_float_sub_c64_r1024", H.subarray([1024, 1024], [1024, 64], [0, 128],
                                                     mpi.ORDER_C, H.named("FLOAT")), 4))
    out.append(("2d_float_sub_c256_r1024", H.subarray([1024, 1024], [1024, 256], [0, 512],
                                                      mpi.ORDER_C, H.named("FLOAT")), 4))
    out.append(("3d_float_sub_c64", H.subarray([256, 256, 256], [256, 256, 64], [0, 0, 64],
                                               mpi.ORDER_C, H.named("FLOAT")), 1))
    out.append(("3d_float_sub_c8", H.subarray([256, 256, 256], [256, 256, 8], [0, 0, 8],
                                              mpi.ORDER_C, H.named("FLOAT")), 1))
    out.append(("3d_double_halo_face_x", H.subarray([260, 260, 260], [256, 256, 2], [2, 2, 2],
                                                    mpi.ORDER_C, H.named("DOUBLE")), 1))
    out.append(("3d_byte_v_hv_100cube", H.make_byte_v_hv((100, 100, 100), (200, 200, 200)), 1))
    return out


def _events():
    import torch

    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def test_reference_kernels_match_tempi_and_oracle(cuda, mpi_init, ref):
    import torch

    results = []
    for name, ty, incount in cases():
        ty.commit()
        o = ty.o
        sb = R.canonicalize(o)
        assert sb.ndims in (2, 3), (name, sb)
        src_np = H.splitmix_bytes(o.extent * incount + 64, 3)
        src = torch.from_numpy(src_np).cuda()
        p_ref = torch.zeros(o.size * incount, dtype=torch.uint8, device="cuda")
        p_tempi = torch.zeros_like(p_ref)
        torch.cuda.synchronize()
        assert ref_launch(ref, sb, 0, src.data_ptr(), p_ref.data_ptr(), incount) == 0
        err, d = mpi.describe(ty.h)
        assert err == 0
        _lib.check(_lib.tempi().tempi_pack(ctypes.byref(d), src.data_ptr(), incount,
                                            p_tempi.data_ptr(), None, None))
        torch.cuda.synchronize()
        want = T.pack(o, src_np, incount) if o.size * incount < (1 << 24) else None
        a, b = p_ref.cpu().numpy(), p_tempi.cpu().numpy()
        assert a.tobytes() == b.tobytes(), name
        if want is not None:
            assert a.tobytes() == want.tobytes(), name
        # unpack parity into 0xAA-filled buffers
        u_ref = torch.full_like(src, 0xAA)
        u_tempi = torch.full_like(src, 0xAA)
        assert ref_launch(ref, sb, 1, u_ref.data_ptr(), p_ref.data_ptr(), incount) == 0
        _lib.check(_lib.tempi().tempi_unpack(ctypes.byref(d), p_tempi.data_ptr(), incount,
                                              u_tempi.data_ptr(), None, None))
        torch.cuda.synchronize()
        assert torch.equal(u_ref, u_tempi), name

        # timing, same stream, 10 launches each after a warm-up
        times = {}
        for who in ("reference", "tempi"):
            for unpack in (0, 1):
                def go():
                    if who == "reference":
                        assert ref_launch(ref, sb, unpack, (u_ref if unpack else src).data_ptr(),
                                          p_ref.data_ptr(), incount) == 0
                    elif unpack:
                        _lib.check(_lib.tempi().tempi_unpack(ctypes.byref(d), p_tempi.data_ptr(),
                                                              incount, u_tempi.data_ptr(), None, None))
                    else:
                        _lib.check(_lib.tempi().tempi_pack(ctypes.byref(d), src.data_ptr(), incount,
                                                            p_tempi.data_ptr(), None, None))
                go()
                e0, e1 = _events()
                e0.record()
                for _ in range(10):
                    go()
                e1.record()
                e1.synchronize()
                times[(who, unpack)] = e0.elapsed_time(e1) / 10
        alg = 2 * o.size * incount
        results.append({
            "case": name, "packed_bytes": o.size * incount, "ref_ndims": sb.ndims,
            "ref_pack_us": round(1e3 * times[("reference", 0)], 2),
            "tempi_pack_us": round(1e3 * times[("tempi", 0)], 2),
            "ref_unpack_us": round(1e3 * times[("reference", 1)], 2),
            "tempi_unpack_us": round(1e3 * times[("tempi", 1)], 2),
            "ref_pack_gbs": round(alg / times[("reference", 0)] / 1e6, 1),
            "tempi_pack_gbs": round(alg / times[("tempi", 0)] / 1e6, 1),
            "pack_speedup": round(times[("reference", 0)] / times[("tempi", 0)], 2),
            "unpack_speedup": round(times[("reference", 1)] / times[("tempi", 1)], 2),
        })
    print(json.dumps(results, indent=1))
    out = os.environ.get("TEMPI_RESULTS_DIR", "")
    if out and os.path.isdir(out):
        with open(os.path.join(out, "ref_vs_tempi.json"), "w") as f:
            json.dump(results, f, indent=1)


def test_reference_kernels_misbehave_where_documented(cuda, mpi_init, ref):
    """The reference chooses its word size from the block length and start
    offset only (pack_kernels.cuh:129-157): with an 8-byte block at a 12-byte
    stride it issues misaligned 8-byte accesses.  That case is left out of
    the parity cases above and is not run here (a misaligned access would
    fault the GPU); this test only shows, on the host, that the reference's
    word-size rule would pick 8 for it while TEMPI's proof picks 4."""
    o = T.vector(64, 8, 12, T.BYTE)
    sb = R.canonicalize(o)
    assert sb.counts[0] == 8 and sb.strides[1] == 12
    ref_w = next(w for w in (8, 6, 4, 3, 2, 1) if sb.counts[0] % w == 0 and sb.start % w == 0)
    assert ref_w == 8
    ty = H.vector(64, 8, 12, H.named()).commit()
    err, d = mpi.describe(ty.h)
    assert err == 0 and d.align == 4


def test_reference_kernels_on_the_sweep(cuda, mpi_init, ref):
    """Every point of the benchmark's strided sweep at its benchmark incount:
    the reference's packer (its pack_2d/pack_3d kernels, or for a contiguous
    type its Packer1D's cudaMemcpyAsync) against the kernel the interposer
    runs (the learned pick), on the same device buffers.  Both write the same
    bytes; both are timed alike (the L2 flushed before every launch, CUDA
    events around it, median of 5; event pair and launch overhead included in
    both).  The sweep's pitches and extents are
    multiples of 16 B and its buffers 256-B aligned, so the reference's word
    size (chosen from block length and start only) is safe on every point.
    Results go to $TEMPI_RESULTS_DIR/ref_kernels_sweep.json when set."""
    import statistics
    import sys

    import torch

    sys.path.insert(0, ROOT)
    from bench import learned_configs, sweep_points

    lib = _lib.tempi()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    rows = []
    for label, sizes, subs, starts, incount in sweep_points():
        o = T.subarray(sizes, subs, starts, T.ORDER_C, T.FLOAT)
        sb = R.canonicalize(o)
        t = mpi.Type_create_subarray(sizes, subs, starts, mpi.ORDER_C, mpi.FLOAT)
        assert mpi.Type_commit(t) == 0
        err, d = mpi.describe(t)
        assert err == 0
        cp, cu = learned_configs(lib, d, incount)
        src = torch.randint(0, 256, (o.extent * incount,), dtype=torch.uint8, device="cuda")
        p_ref = torch.zeros(o.size * incount, dtype=torch.uint8, device="cuda")
        p_tempi = torch.zeros_like(p_ref)
        u_ref = torch.full_like(src, 0xAA)
        u_tempi = torch.full_like(src, 0xAA)
        contiguous = sb.ndims <= 1

        def launch(who, unpack):
            if who == "tempi":
                if unpack:
                    _lib.check(lib.tempi_unpack(ctypes.byref(d), p_tempi.data_ptr(), incount,
                                                u_tempi.data_ptr(), ctypes.byref(cu) if cu else None,
                                                None))
                else:
                    _lib.check(lib.tempi_pack(ctypes.byref(d), src.data_ptr(), incount,
                                              p_tempi.data_ptr(), ctypes.byref(cp) if cp else None,
                                              None))
            elif contiguous:  # Packer1D: one cudaMemcpyAsync of the packed bytes
                off = sb.start if sb.ndims == 1 else 0
                if unpack:
                    u_ref[off: off + p_ref.numel()].copy_(p_ref)
                else:
                    p_ref.copy_(src[off: off + p_ref.numel()])
            else:
                assert ref_launch(ref, sb, unpack, (u_ref if unpack else src).data_ptr(),
                                  p_ref.data_ptr(), incount) == 0

        times = {}
        for who in ("reference", "tempi"):
            for unpack in (0, 1):
                launch(who, unpack)
                ts = []
                for _ in range(5):
                    flush.fill_(1)  # evict the L2, then read back so its lines are clean
                    flush.view(torch.int64).sum()
                    e0, e1 = _events()
                    e0.record()
                    launch(who, unpack)
                    e1.record()
                    e1.synchronize()
                    ts.append(e0.elapsed_time(e1))
                times[(who, unpack)] = statistics.median(ts)
        torch.cuda.synchronize()
        assert torch.equal(p_ref, p_tempi), label
        assert torch.equal(u_ref, u_tempi), label
        mpi.Type_free(t)
        alg = 2 * o.size * incount
        rows.append({
            "point": label, "incount": incount, "packed_bytes": o.size * incount,
            "reference": "Packer1D cudaMemcpyAsync" if contiguous else f"pack_{sb.ndims}d",
            "ref_pack_gbs": round(alg / times[("reference", 0)] / 1e6, 1),
            "ref_unpack_gbs": round(alg / times[("reference", 1)] / 1e6, 1),
            "tempi_pack_gbs": round(alg / times[("tempi", 0)] / 1e6, 1),
            "tempi_unpack_gbs": round(alg / times[("tempi", 1)] / 1e6, 1),
            "pack_speedup": round(times[("reference", 0)] / times[("tempi", 0)], 2),
            "unpack_speedup": round(times[("reference", 1)] / times[("tempi", 1)], 2),
        })
    print(json.dumps(rows, indent=1))
    out = os.environ.get("TEMPI_RESULTS_DIR", "")
    if out and os.path.isdir(out):
        with open(os.path.join(out, "ref_kernels_sweep.json"), "w") as f:
            json.dump(rows, f, indent=1)


def test_reference_kernels_on_the_halo(cuda, mpi_init, ref):
    """The 256^3 grid of doubles at radius 2: its 26 send regions packed by
    the reference's packer (one pack_3d launch per region, as the reference's
    MPI_Pack runs them, without the synchronisation after each), by this
    library's plain kernels (one launch per region, the learned picks) and by
    one batched launch, on the same buffers; and the oracle's C walker on one
    host core over the same regions (the CPU baseline).  All write the same
    bytes.  Each GPU sequence is timed with CUDA events around its launches,
    the L2 flushed before each, median of 5.  Results go to
    $TEMPI_RESULTS_DIR/halo_ref_kernels.json when set."""
    import statistics
    import sys
    import time

    import torch

    from oracle import walker as W
    from tempi_b200 import halo

    sys.path.insert(0, ROOT)
    from bench import learned_configs

    lib = _lib.tempi()
    g = halo.Grid((256, 256, 256), 2)
    gen = torch.Generator(device="cuda").manual_seed(33)
    data = torch.randint(0, 256, (g.nbytes,), dtype=torch.uint8, device="cuda", generator=gen)
    packs = {k: torch.zeros(g.packed_bytes, dtype=torch.uint8, device="cuda")
             for k in ("reference", "plain", "batched")}
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    offs = g.offsets()
    sizes = [g.alloc[2], g.alloc[1], g.alloc[0]]
    plan = []
    for d in halo.directions():
        subs, starts = g.region_shape[(d, False)]
        o = T.subarray(sizes, subs, starts, T.ORDER_C, T.named(8))
        sb = R.canonicalize(o)
        assert sb.ndims == 3  # no region spans a full row of the grid
        # the reference's word size (from block and start) divides every
        # stride and packed offset here, so its kernel is correct
        assert sb.strides[1] % 8 == 0 and sb.strides[2] % 8 == 0 and offs[d] % 8 == 0
        err, desc = mpi.describe(g.send[d])
        assert err == 0
        cp, _ = learned_configs(lib, desc, 1)
        plan.append((d, o, sb, desc, cp))
    batch = halo.HaloBatch([g], [data.data_ptr()], [packs["batched"].data_ptr()])

    def run(who):
        p = packs[who]
        if who == "batched":
            batch.launch()
            return
        for d, _, sb, desc, cp in plan:
            dst = p.data_ptr() + offs[d]
            if who == "reference":
                assert ref_launch(ref, sb, 0, data.data_ptr(), dst, 1) == 0
            else:
                _lib.check(lib.tempi_pack(ctypes.byref(desc), data.data_ptr(), 1, dst,
                                          ctypes.byref(cp) if cp else None, None))

    times = {}
    for who in ("reference", "plain", "batched"):
        run(who)
        ts = []
        for _ in range(5):
            flush.fill_(1)
            flush.view(torch.int64).sum()
            e0, e1 = _events()
            e0.record()
            run(who)
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) * 1e3)
        times[who] = statistics.median(ts)
    torch.cuda.synchronize()
    assert torch.equal(packs["reference"], packs["plain"])
    assert torch.equal(packs["batched"], packs["plain"])
    batch.close()

    host = data.cpu().numpy()
    walkers = [(d, W.Walker(o)) for d, o, _, _, _ in plan]
    cpu = []
    for _ in range(5):
        t0 = time.perf_counter()
        out = np.concatenate([w.pack(host, 1, nthreads=1) for _, w in walkers])
        cpu.append((time.perf_counter() - t0) * 1e6)
    assert np.array_equal(out, packs["plain"].cpu().numpy())
    row = {"grid": "256^3 doubles, radius 2, 26 regions", "packed_bytes": g.packed_bytes,
           "reference_26_launches_us": round(times["reference"], 1),
           "tempi_26_launches_us": round(times["plain"], 1),
           "tempi_batched_us": round(times["batched"], 1),
           "oracle_c_walker_1_core_us": round(statistics.median(cpu), 1)}
    print(json.dumps(row))
    res = os.environ.get("TEMPI_RESULTS_DIR", "")
    if res and os.path.isdir(res):
        with open(os.path.join(res, "halo_ref_kernels.json"), "w") as f:
            json.dump(row, f, indent=1)
