"""Dispatch on CPU: the restated table model's interpolation against the
reference's known answers (test/measure_system.cpp:13-92) and the oracle's
restatement, and the features of a layout."""
import ctypes

import numpy as np

from oracle import interp as I
from tempi_b200 import _lib


def _interp(table, bytes_, block=0):
    a = np.ascontiguousarray(table, np.float64)
    rows, cols = (a.shape[0], 0) if a.ndim == 1 else a.shape
    return _lib.tempi().tempi_table_interp(a.ctypes.data, rows, cols, bytes_, block)


def test_table_1d_known_answers():
    v = [2, 4, 8, 16]
    assert [_interp(v, b) for b in (1, 2, 3, 5, 7)] == [2, 4, 6, 10, 14]


def test_table_2d_known_answers():
    a = [[14, 18, 22], [16, 20, 24]]
    cases = {(64, 1): 14, (160, 1): 15, (256, 1): 16, (64, 2): 18, (256, 2): 20,
             (64, 3): 20, (64, 4): 22, (160, 3): 21, (512, 1): 32, (512, 3): 44}
    for (b, s), want in cases.items():
        assert abs(_interp(a, b, s) - want) < 1e-4, (b, s)


def test_table_model_matches_oracle_restatement():
    rng = np.random.default_rng(0)
    a = rng.uniform(1, 100, (6, 10))
    v = list(rng.uniform(1, 100, 12))
    for _ in range(300):
        b = int(rng.integers(1, 1 << 26))
        s = int(rng.integers(1, 513))
        assert abs(_interp(a, b, s) - I.interp_2d(a.tolist(), b, s)) <= 1e-3 * abs(I.interp_2d(a.tolist(), b, s))
        assert abs(_interp(v, b) - I.interp_time(v, b)) <= 1e-3 * abs(I.interp_time(v, b))


def test_features_of_a_layout():
    d = _lib.Desc.make(0, 1 << 20, 64, [1024], [512])
    f = (ctypes.c_float * 12)()
    assert _lib.tempi().tempi_features(ctypes.byref(d), 2, 0, 1, f) == 0
    x = np.frombuffer(f, np.float32)
    assert abs(x[1] - 6 / 32) < 1e-6           # log2 block
    assert abs(x[6] - np.log2(2 * 64 * 1024) / 32) < 1e-6  # log2 total bytes
    assert abs(x[7] - 1 / 32) < 1e-6            # log2 incount
    assert x[9] == 0 and x[10] == 1             # typed on device, packed on host
