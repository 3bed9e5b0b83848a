"""Failures injected on the host, on the GPU send paths: an intermediate
slab allocation that fails (TEMPI_TEST_FAIL_SLAB, the n-th allocation from
the knob on), and the underlying MPI returning an error from MPI_Send,
MPI_Start, MPI_Test or MPI_Recv (the stand-in library's minimpi_fail_nth
hook).  Where the reference exits the process (include/cuda_runtime.hpp:
13-18, include/logging.hpp:70-76), each call here returns the MPI error,
sends nothing it should not, leaks no slab, and leaves the library usable:
the next transfer is bit-exact.  No GPU fault, trap or hang is involved."""
import ctypes
import os

import numpy as np
import pytest

from tempi_b200 import _lib, mpi

from . import helpers as H

pytestmark = pytest.mark.gpu

ERR_NO_MEM = 34


def _fail_lib(call, n):
    lib = _lib.minimpi()
    lib.minimpi_fail_nth.argtypes = [ctypes.c_char_p, ctypes.c_int]
    assert lib.minimpi_fail_nth(call.encode(), n) == 0


@pytest.fixture
def method():
    """Force a send method for the test, and clear every knob afterwards."""
    knobs = ("TEMPI_DATATYPE_DEVICE", "TEMPI_DATATYPE_STAGED", "TEMPI_DATATYPE_ONESHOT",
             "TEMPI_TEST_FAIL_SLAB")

    def set_method(name):
        for k in knobs[:3]:
            os.environ.pop(k, None)
        os.environ["TEMPI_DATATYPE_" + name] = ""
        _lib.tempi().tempi_reload_env()

    yield set_method
    for k in knobs:
        os.environ.pop(k, None)
    _lib.tempi().tempi_reload_env()
    _fail_lib("", 0)


def _arm_slab_failure(n):
    os.environ["TEMPI_TEST_FAIL_SLAB"] = str(n)
    _lib.tempi().tempi_reload_env()
    os.environ.pop("TEMPI_TEST_FAIL_SLAB", None)  # a later reload disarms it


def _buffers(t, seed):
    import torch

    src_np = H.splitmix_bytes(t.o.extent, seed)
    return src_np, torch.from_numpy(src_np).cuda(), torch.full((t.o.extent,), 0xAA,
                                                               dtype=torch.uint8, device="cuda")


def _expect(t, src_np):
    from oracle import types as T

    exp = np.full_like(src_np, 0xAA)
    T.unpack(t.o, T.pack(t.o, src_np, 1), exp, 1)
    return exp


def _round_trip_ok(t, seed):
    """A blocking self-send of fresh data arrives bit-exact."""
    import torch

    src_np, src, dst = _buffers(t, seed)
    assert mpi.Send(src.data_ptr(), 1, t.h, tag=9) == 0, _lib.last_error()
    err, _ = mpi.Recv(dst.data_ptr(), 1, t.h, tag=9)
    assert err == 0, _lib.last_error()
    torch.cuda.synchronize()
    assert dst.cpu().numpy().tobytes() == _expect(t, src_np).tobytes()


@pytest.mark.parametrize("name,nth", [("DEVICE", 1), ("ONESHOT", 1), ("STAGED", 1),
                                      ("STAGED", 2)])
def test_send_slab_failure(cuda, mpi_init, method, name, nth):
    """The send's slab (for STAGED: the device one, or the host one after
    it) cannot be had: MPI_Send returns MPI_ERR_NO_MEM, no message is left
    in the library (the next receive gets the next send's data) and every
    slab it took is back."""
    t = H.make_2d_byte_vector(256, 64, 128).commit()
    method(name)
    _round_trip_ok(t, 1)  # warm: slabs of this size now come from the cache
    live = _lib.counter("slab_live_bytes")
    _, src, _ = _buffers(t, 2)
    _arm_slab_failure(nth)
    assert mpi.Send(src.data_ptr(), 1, t.h, tag=9) == ERR_NO_MEM
    assert _lib.counter("slab_live_bytes") == live
    _round_trip_ok(t, 3)
    assert _lib.counter("slab_live_bytes") == live


@pytest.mark.parametrize("name", ["DEVICE", "ONESHOT", "STAGED"])
def test_recv_slab_failure(cuda, mpi_init, method, name):
    """A receive whose slab cannot be had returns MPI_ERR_NO_MEM and leaves
    the message queued: the next receive gets it, bit-exact."""
    import torch

    t = H.make_2d_byte_vector(256, 64, 128).commit()
    method(name)
    _round_trip_ok(t, 4)
    live = _lib.counter("slab_live_bytes")
    src_np, src, dst = _buffers(t, 5)
    assert mpi.Send(src.data_ptr(), 1, t.h, tag=9) == 0
    _arm_slab_failure(1)
    err, _ = mpi.Recv(dst.data_ptr(), 1, t.h, tag=9)
    assert err == ERR_NO_MEM
    assert _lib.counter("slab_live_bytes") == live
    err, _ = mpi.Recv(dst.data_ptr(), 1, t.h, tag=9)
    assert err == 0, _lib.last_error()
    torch.cuda.synchronize()
    assert dst.cpu().numpy().tobytes() == _expect(t, src_np).tobytes()
    assert _lib.counter("slab_live_bytes") == live


@pytest.mark.parametrize("name", ["DEVICE", "STAGED"])
def test_library_send_error(cuda, mpi_init, method, name):
    """The underlying MPI_Send fails after TEMPI packed: MPI_Send returns
    the library's error, the slab comes back, nothing was queued."""
    t = H.make_2d_byte_vector(256, 64, 128).commit()
    method(name)
    _round_trip_ok(t, 6)
    live = _lib.counter("slab_live_bytes")
    _, src, _ = _buffers(t, 7)
    _fail_lib("MPI_Send", 1)
    assert mpi.Send(src.data_ptr(), 1, t.h, tag=9) == mpi.ERR_OTHER
    assert _lib.counter("slab_live_bytes") == live
    _round_trip_ok(t, 8)


def test_isend_start_error_reported_by_wait(cuda, mpi_init, method):
    """MPI_Isend packs and returns; the library's MPI_Start (the managed
    send starts once its pack is done) fails: MPI_Wait returns that error,
    frees the request and its slab, and the next transfer works."""
    t = H.make_2d_byte_vector(256, 64, 128).commit()
    method("DEVICE")
    _round_trip_ok(t, 9)
    live = _lib.counter("slab_live_bytes")
    _, src, _ = _buffers(t, 10)
    _fail_lib("MPI_Start", 1)
    err, req = mpi.Isend(src.data_ptr(), 1, t.h, tag=9)
    assert err == 0, _lib.last_error()
    err = mpi.Wait(req)[0]
    assert err == mpi.ERR_OTHER
    assert _lib.counter("slab_live_bytes") == live
    _round_trip_ok(t, 11)
    assert _lib.counter("slab_live_bytes") == live


def test_irecv_test_error_reported_by_wait(cuda, mpi_init, method):
    """A managed MPI_Irecv whose library MPI_Test fails: MPI_Wait returns
    the error, frees the request and slab; later transfers are exact."""
    t = H.make_2d_byte_vector(256, 64, 128).commit()
    method("DEVICE")
    _round_trip_ok(t, 12)
    live = _lib.counter("slab_live_bytes")
    src_np, src, dst = _buffers(t, 13)
    err, rreq = mpi.Irecv(dst.data_ptr(), 1, t.h, tag=9)
    assert err == 0
    _fail_lib("MPI_Test", 1)
    err = mpi.Wait(rreq)[0]
    assert err == mpi.ERR_OTHER
    _fail_lib("", 0)
    assert _lib.counter("slab_live_bytes") == live
    _round_trip_ok(t, 14)
    assert _lib.counter("slab_live_bytes") == live


def test_library_recv_error(cuda, mpi_init, method):
    """The underlying MPI_Recv fails: TEMPI's MPI_Recv returns it, frees its
    slab, and the queued message is received by the next call."""
    import torch

    t = H.make_2d_byte_vector(256, 64, 128).commit()
    method("DEVICE")
    _round_trip_ok(t, 15)
    live = _lib.counter("slab_live_bytes")
    src_np, src, dst = _buffers(t, 16)
    assert mpi.Send(src.data_ptr(), 1, t.h, tag=9) == 0
    _fail_lib("MPI_Recv", 1)
    err, _ = mpi.Recv(dst.data_ptr(), 1, t.h, tag=9)
    assert err == mpi.ERR_OTHER
    assert _lib.counter("slab_live_bytes") == live
    err, _ = mpi.Recv(dst.data_ptr(), 1, t.h, tag=9)
    assert err == 0
    torch.cuda.synchronize()
    assert dst.cpu().numpy().tobytes() == _expect(t, src_np).tobytes()


def test_slab_cache_is_capped(cuda, mpi_init, method):
    """Freed slabs are kept only up to TEMPI_SLAB_CACHE_MB per memory space,
    and large ones are rounded to 2 MiB, not to a power of two: a 65 MiB +
    1 B message holds 66 MiB while it is in flight and nothing afterwards
    when the cap is 64 MiB."""
    import torch

    os.environ["TEMPI_SLAB_CACHE_MB"] = "64"
    _lib.tempi().tempi_reload_env()
    try:
        method("DEVICE")
        n = (65 << 20) + 1
        t = mpi.Type_vector(n, 1, 2, mpi.BYTE)  # 65 MiB + 1 B of 1-byte blocks
        assert mpi.Type_commit(t) == 0
        ext = 2 * n - 1
        src = torch.randint(0, 256, (ext,), dtype=torch.uint8, device="cuda")
        dst = torch.zeros_like(src)
        held0 = _lib.counter("slab_bytes")
        cached0 = _lib.counter("slab_cached_bytes")
        assert mpi.Send(src.data_ptr(), 1, t, tag=3) == 0
        # the eager send is done; its slab went back, above the cap: released
        assert _lib.counter("slab_cached_bytes") <= cached0
        err, _ = mpi.Recv(dst.data_ptr(), 1, t, tag=3)
        assert err == 0
        torch.cuda.synchronize()
        assert torch.equal(dst[::2], src[::2])
        # neither message's slab stayed behind (blocks cached before the cap
        # was lowered may remain, but nothing was added to them)
        assert _lib.counter("slab_cached_bytes") <= cached0
        assert _lib.counter("slab_bytes") <= held0
        mpi.Type_free(t)
    finally:
        os.environ.pop("TEMPI_SLAB_CACHE_MB", None)
        _lib.tempi().tempi_reload_env()
