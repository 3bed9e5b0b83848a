"""Self-sends of strided device objects through the interposed
MPI_Send/MPI_Recv/MPI_Isend/MPI_Irecv/MPI_Wait, by each transfer method
(the self-send workload at small sizes).  The reference only checks that these
complete (test/isend.cu, test/send.cpp); here every received byte is
compared with the oracle and gap bytes must keep their 0xAA fill."""
import os

import numpy as np
import pytest

from oracle import types as T
from tempi_b200 import _lib, mpi

from . import helpers as H

pytestmark = pytest.mark.gpu

METHODS = {"DEVICE": "TEMPI_DATATYPE_DEVICE", "ONESHOT": "TEMPI_DATATYPE_ONESHOT",
           "STAGED": "TEMPI_DATATYPE_STAGED"}


@pytest.fixture
def method(request):
    var = METHODS[request.param]
    os.environ[var] = ""
    _lib.tempi().tempi_reload_env()
    yield request.param
    os.environ.pop(var, None)
    _lib.tempi().tempi_reload_env()


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def expected(ty, src, count):
    exp = np.full_like(src, 0xAA)
    T.unpack(ty.o, T.pack(ty.o, src, count), exp, count)
    return exp


def types():
    return [
        H.vector(300, 3, 17, H.named("BYTE")),
        H.subarray([40, 30, 20], [10, 12, 6], [3, 4, 5], mpi.ORDER_C, H.named("FLOAT")),
        H.make_byte_v_hv((64, 9, 5), (128, 16, 8)),
        H.vector(64, 1024, 2048, H.named("FLOAT")),
    ]


@pytest.mark.parametrize("method", list(METHODS), indirect=True)
def test_blocking_self_send(cuda, mpi_init, method):
    import torch

    before = _lib.counter("send_" + method.lower())
    for ty in types():
        ty.commit()
        count = 2
        src_np = H.splitmix_bytes(ty.o.extent * count, 11)
        src, dst = dev(src_np), dev(np.full_like(src_np, 0xAA))
        torch.cuda.synchronize()
        assert mpi.Send(src.data_ptr(), count, ty.h) == 0, _lib.last_error()
        err, st = mpi.Recv(dst.data_ptr(), count, ty.h)
        assert err == 0, _lib.last_error()
        assert mpi.Get_count(st, ty.h) == count
        assert dst.cpu().numpy().tobytes() == expected(ty, src_np, count).tobytes(), ty.name
    assert _lib.counter("send_" + method.lower()) == before + len(types())


@pytest.mark.parametrize("method", list(METHODS), indirect=True)
@pytest.mark.parametrize("recv_first", [True, False])
def test_nonblocking_self_send(cuda, mpi_init, method, recv_first):
    import torch

    for ty in types():
        ty.commit()
        count = 3
        src_np = H.splitmix_bytes(ty.o.extent * count, 12)
        src, dst = dev(src_np), dev(np.full_like(src_np, 0xAA))
        torch.cuda.synchronize()
        if recv_first:
            e1, rr = mpi.Irecv(dst.data_ptr(), count, ty.h, tag=7)
            e2, rs = mpi.Isend(src.data_ptr(), count, ty.h, tag=7)
        else:
            e2, rs = mpi.Isend(src.data_ptr(), count, ty.h, tag=7)
            e1, rr = mpi.Irecv(dst.data_ptr(), count, ty.h, tag=7)
        assert (e1, e2) == (0, 0), _lib.last_error()
        assert rr & 0x40000000 and rs & 0x40000000  # managed requests
        err, r, st = mpi.Wait(rr)
        assert err == 0 and r == mpi.REQUEST_NULL, _lib.last_error()
        err, r, _ = mpi.Wait(rs)
        assert err == 0 and r == mpi.REQUEST_NULL
        assert dst.cpu().numpy().tobytes() == expected(ty, src_np, count).tobytes(), ty.name


def test_tags_match_in_order(cuda, mpi_init):
    import torch

    ty = H.vector(50, 4, 9, H.named("BYTE")).commit()
    a_np, b_np = H.splitmix_bytes(ty.o.extent, 1), H.splitmix_bytes(ty.o.extent, 2)
    a, b = dev(a_np), dev(b_np)
    ra, rb = dev(np.full_like(a_np, 0xAA)), dev(np.full_like(a_np, 0xAA))
    torch.cuda.synchronize()
    assert mpi.Send(a.data_ptr(), 1, ty.h, tag=1) == 0
    assert mpi.Send(b.data_ptr(), 1, ty.h, tag=2) == 0
    assert mpi.Recv(rb.data_ptr(), 1, ty.h, tag=2)[0] == 0
    assert mpi.Recv(ra.data_ptr(), 1, ty.h, tag=1)[0] == 0
    assert ra.cpu().numpy().tobytes() == expected(ty, a_np, 1).tobytes()
    assert rb.cpu().numpy().tobytes() == expected(ty, b_np, 1).tobytes()


def test_wait_without_sender_times_out(cuda, mpi_init):
    """Failure detection without a GPU fault: a receive whose send never
    comes makes MPI_Wait return an error after TEMPI_WAIT_TIMEOUT_S instead
    of spinning forever; the context stays usable afterwards."""
    import torch

    os.environ["TEMPI_WAIT_TIMEOUT_S"] = "0.5"
    _lib.tempi().tempi_reload_env()
    try:
        ty = H.vector(20, 2, 5, H.named("BYTE")).commit()
        dst = dev(np.zeros(ty.o.extent, np.uint8))
        err, rr = mpi.Irecv(dst.data_ptr(), 1, ty.h, tag=99)
        assert err == 0
        err, r, _ = mpi.Wait(rr)
        assert err == mpi.ERR_OTHER and r == mpi.REQUEST_NULL
        assert "gave up" in _lib.last_error()
    finally:
        os.environ.pop("TEMPI_WAIT_TIMEOUT_S")
        _lib.tempi().tempi_reload_env()
    # still usable
    test_tags_match_in_order(torch.device("cuda"), mpi_init)


@pytest.mark.parametrize("mode", ["STAGED", "AUTO", "NONE"])
def test_contiguous_device_send(cuda, mpi_init, mode):
    """Contiguous device buffers (named MPI_FLOAT and MPI_BYTE, a derived
    contiguous type): TEMPI_CONTIGUOUS_STAGED stages every send and receive
    through host memory (reference SendRecv1DStaged, sender.cpp:34-61),
    TEMPI_CONTIGUOUS_AUTO stages when the measured tables say it is faster
    (SendRecv1D, sender.cpp:63-88), and without either the library sends the
    device buffer as it is.  Every received byte must match."""
    import torch

    var = {"STAGED": "TEMPI_CONTIGUOUS_STAGED", "AUTO": "TEMPI_CONTIGUOUS_AUTO"}.get(mode)
    if var:
        os.environ[var] = ""
    _lib.tempi().tempi_reload_env()
    try:
        dbl = H.contiguous(77, H.named("DOUBLE")).commit()
        for t, count, size in ((mpi.FLOAT, 3000, 4), (dbl.h, 5, 616), (mpi.BYTE, 1 << 20, 1)):
            src_np = H.splitmix_bytes(count * size, count)
            src, dst = dev(src_np), dev(np.zeros_like(src_np))
            torch.cuda.synchronize()
            s0 = _lib.counter("send_contig_staged")
            r0 = _lib.counter("recv_contig_staged")
            assert mpi.Send(src.data_ptr(), count, t, tag=7) == 0
            assert mpi.Recv(dst.data_ptr(), count, t, tag=7)[0] == 0
            assert dst.cpu().numpy().tobytes() == src_np.tobytes()
            ds = _lib.counter("send_contig_staged") - s0
            dr = _lib.counter("recv_contig_staged") - r0
            if mode == "STAGED":
                assert ds == 1 and dr == 1
            elif mode == "NONE":
                assert ds == 0 and dr == 0
            else:  # the same model decides both sides of the same byte count
                assert ds == dr and ds in (0, 1)
    finally:
        if var:
            os.environ.pop(var, None)
        _lib.tempi().tempi_reload_env()


def test_non_overtaking_across_managed_and_library_sends(cuda, mpi_init):
    """MPI's non-overtaking rule with one destination and one tag: a strided
    Isend (packed by a kernel first, so its library send is deferred), then
    a plain byte Isend, then another strided Isend.  Received in that order
    -- and waited on out of order -- each message lands in its own
    receive."""
    import torch

    vec = H.vector(200, 3, 7, H.named("BYTE")).commit()
    a_np, c_np = H.splitmix_bytes(vec.o.extent, 1), H.splitmix_bytes(vec.o.extent, 3)
    b_np = H.splitmix_bytes(57, 2)
    a, b, c = dev(a_np), dev(b_np), dev(c_np)
    ra = dev(np.full_like(a_np, 0xAA))
    rb = dev(np.zeros_like(b_np))
    rc = dev(np.full_like(c_np, 0xAA))
    torch.cuda.synchronize()
    e1, q1 = mpi.Isend(a.data_ptr(), 1, vec.h, tag=5)
    e2, q2 = mpi.Isend(b.data_ptr(), 57, mpi.BYTE, tag=5)
    e3, q3 = mpi.Isend(c.data_ptr(), 1, vec.h, tag=5)
    e4, p1 = mpi.Irecv(ra.data_ptr(), 1, vec.h, tag=5)
    e5, p2 = mpi.Irecv(rb.data_ptr(), 57, mpi.BYTE, tag=5)
    e6, p3 = mpi.Irecv(rc.data_ptr(), 1, vec.h, tag=5)
    assert (e1, e2, e3, e4, e5, e6) == (0,) * 6
    for q in (q3, q1, q2, p3, p2, p1):  # out of order on purpose
        assert mpi.Wait(q)[0] == 0
    assert ra.cpu().numpy().tobytes() == expected(vec, a_np, 1).tobytes()
    assert rb.cpu().numpy().tobytes() == b_np.tobytes()
    assert rc.cpu().numpy().tobytes() == expected(vec, c_np, 1).tobytes()
