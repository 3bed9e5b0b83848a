"""The learned dispatch with the committed model (tempi_b200/models/):
the harness measures every eligible candidate, the dispatcher picks among
them, MPI_Pack uses the pick and stays bit-exact, and on fresh layouts the
model's picks cost less in total than the fixed rules' (what the network
gains over the method without it)."""
import ctypes
import os

import numpy as np
import pytest

from oracle import types as T
from tempi_b200 import _lib, dispatch_train as DT, mpi

from . import helpers as H

pytestmark = pytest.mark.gpu

MODEL = os.path.join(DT.MODELS, DT.MODEL_FILE)
TABLE = os.path.join(DT.MODELS, DT.TABLE_FILE)


@pytest.fixture(scope="module")
def model(cuda, mpi_init):
    assert os.path.exists(MODEL), "the trained cost model is missing"
    _lib.check(_lib.tempi().tempi_dispatch_load(MODEL.encode(), TABLE.encode()))


def test_measure_covers_eligible_candidates(model):
    """Packs ([0..9]) and unpacks ([10..19]) are timed apart for every
    eligible configuration, transfers by the three methods ([20..22]), and
    the fixed rules' pack and unpack ([23], [24])."""
    lib = _lib.tempi()
    t = (ctypes.c_float * DT.N_MEAS)()
    d = _lib.Desc.make(4, 1 << 22, 1000, [2000], [2048])
    _lib.check(lib.tempi_measure(ctypes.byref(d), 1, 0, 0, 3, 2, t))
    v = np.frombuffer(t, np.float32)
    assert np.isfinite(v).all() and (v > 0).all(), v  # 1000-B rows: all eligible
    d = _lib.Desc.make(0, 1 << 20, 1 << 20, [], [])  # one contiguous block
    _lib.check(lib.tempi_measure(ctypes.byref(d), 1, 0, 0, 1, 2, t))
    v = np.frombuffer(t, np.float32)
    for lo in (DT.PACK, DT.UNPACK):  # the word and staged kernels suit one block
        assert np.isfinite(v[lo:lo + 3]).all() and np.isnan(v[lo + 3:lo + 8]).all()
        assert np.isfinite(v[lo + 8:lo + 10]).all()
    assert np.isnan(v[DT.METH:DT.METH + 3]).all()
    assert np.isfinite(v[DT.FIXED_PACK]) and np.isfinite(v[DT.FIXED_UNPACK])


def test_choice_is_eligible_and_pack_stays_exact(model):
    rng = np.random.default_rng(11)
    before = _lib.counter("dispatch_miss")
    for _ in range(20):
        ty = H.random_type(rng).commit()  # MPI_Type_commit runs the model
        err, d = mpi.describe(ty.h)
        if err:
            continue
        pc, uc, mi = ctypes.c_int(-2), ctypes.c_int(-2), ctypes.c_int(0)
        pred = (ctypes.c_float * DT.N_OUT)()
        _lib.check(_lib.tempi().tempi_dispatch_choose(ctypes.byref(d), 2, 0, 0, 0,
                                                       ctypes.byref(pc), ctypes.byref(uc),
                                                       ctypes.byref(mi), pred, None))
        assert 0 <= pc.value < DT.N_CFG and 0 <= uc.value < DT.N_CFG and 1 <= mi.value <= 3
        assert np.isfinite(np.frombuffer(pred, np.float32)).all()
        import torch

        src_np = H.splitmix_bytes(max(ty.o.extent * 2, 1) + 64, 3)
        src = torch.from_numpy(src_np).cuda()
        out = torch.zeros(max(ty.o.size * 2, 1), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        e, pos = mpi.Pack(src.data_ptr(), 2, ty.h, out.data_ptr(), out.numel())
        assert e == 0
        assert out.cpu().numpy()[:pos].tobytes() == T.pack(ty.o, src_np, 2).tobytes()
    assert _lib.counter("dispatch_miss") > before


def test_learned_beats_fixed_rules_on_fresh_layouts(model):
    """Fresh layouts (a seed the model never saw), device and host buffers:
    the learned pack and unpack picks together cost less than the fixed
    rules' and stay within 10 % of exhaustive search."""
    lib = _lib.tempi()
    rng = np.random.default_rng(4242)
    t = (ctypes.c_float * DT.N_MEAS)()
    L, F, B = [], [], []
    while len(B) < 120:
        d, incount, th, ph = DT.random_layout(rng)
        if DT.span_of(d, incount) > (1 << 30) or (th and DT.span_of(d, incount) > (16 << 20)):
            continue
        _lib.check(lib.tempi_measure(ctypes.byref(d), incount, int(th), int(ph), 1, 2, t))
        pc, uc, mi = ctypes.c_int(-1), ctypes.c_int(-1), ctypes.c_int(0)
        _lib.check(lib.tempi_dispatch_choose(ctypes.byref(d), incount, int(th), int(ph), 0,
                                              ctypes.byref(pc), ctypes.byref(uc),
                                              ctypes.byref(mi), None, None))
        v = np.frombuffer(t, np.float32)
        tp, tu = v[DT.PACK:DT.PACK + DT.N_CFG], v[DT.UNPACK:DT.UNPACK + DT.N_CFG]
        B.append(np.nanmin(tp) + np.nanmin(tu))
        L.append(tp[pc.value] + tu[uc.value])
        F.append(v[DT.FIXED_PACK] + v[DT.FIXED_UNPACK])
    L, F, B = map(np.array, (L, F, B))
    learned, fixed = L.sum() / B.sum() - 1, F.sum() / B.sum() - 1
    print(f"total-time regret: learned {learned:.3f}, fixed rules {fixed:.3f}")
    assert learned < fixed
    assert learned < 0.10


def test_layout_cache_serves_a_new_handle_of_a_known_shape(model):
    """A second handle of a layout committed before takes the choices made
    for the first (no inference, no measurement): MPI_Type_commit of the
    same shape again counts only dispatch hits, and the pack through the new
    handle is still exact."""
    import torch

    def make():
        return mpi.Type_create_subarray([64, 64, 64], [64, 48, 24], [0, 5, 7],
                                        mpi.ORDER_C, mpi.FLOAT)

    t1 = make()
    assert mpi.Type_commit(t1) == 0
    miss0, hit0 = _lib.counter("dispatch_miss"), _lib.counter("dispatch_hit")
    t2 = make()
    assert mpi.Type_commit(t2) == 0
    assert _lib.counter("dispatch_miss") == miss0
    assert _lib.counter("dispatch_hit") > hit0
    o = T.subarray([64, 64, 64], [64, 48, 24], [0, 5, 7], T.ORDER_C, T.FLOAT)
    src_np = H.splitmix_bytes(o.extent + 64, 12)
    src = torch.from_numpy(src_np).cuda()
    out = torch.zeros(o.size, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    e, pos = mpi.Pack(src.data_ptr(), 1, t2, out.data_ptr(), out.numel())
    assert e == 0 and pos == o.size
    assert out.cpu().numpy().tobytes() == T.pack(o, src_np, 1).tobytes()
    mpi.Type_free(t1)
    mpi.Type_free(t2)


def test_host_layouts_outside_training_are_measured(model):
    """A host-resident layout beyond the model's training range (here 4 MiB
    packed from a 64 MiB pinned span: 262,144 rows of 16 B, 256 B apart) is
    not left to the model's extrapolation: MPI_Pack's first use times the
    candidates (dispatch_measured moves once for the pack and the unpack
    together), picks an eligible one, and both directions stay exact."""
    import torch

    t = mpi.Type_vector(262144, 4, 64, mpi.FLOAT)
    assert mpi.Type_commit(t) == 0
    err, d = mpi.describe(t)
    assert err == 0 and d.size == 4 << 20
    span = d.extent
    src_np = H.splitmix_bytes(span, 17)
    src = torch.from_numpy(src_np).pin_memory()
    out = torch.zeros(d.size, dtype=torch.uint8).pin_memory()
    m0 = _lib.counter("dispatch_measured")
    e, pos = mpi.Pack(src.data_ptr(), 1, t, out.data_ptr(), out.numel())
    assert e == 0 and pos == d.size
    want = T.pack(T.vector(262144, 4, 64, T.FLOAT), src_np, 1)
    assert out.numpy().tobytes() == want.tobytes()
    assert _lib.counter("dispatch_measured") == m0 + 1
    back = torch.full_like(src, 0xAA).pin_memory()
    e, _ = mpi.Unpack(out.data_ptr(), out.numel(), back.data_ptr(), 1, t)
    assert e == 0
    exp = np.full(span, 0xAA, np.uint8)
    T.unpack(T.vector(262144, 4, 64, T.FLOAT), want, exp, 1)
    assert back.numpy().tobytes() == exp.tobytes()
    # the pack's measurement chose the unpack too
    assert _lib.counter("dispatch_measured") == m0 + 1
    mpi.Type_free(t)
