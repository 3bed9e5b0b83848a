"""ORACLE -- test infrastructure only.

Restatement of the reference's measured-table interpolation, the method
model that the learned dispatch replaces:

* ``interp_time``  src/internal/measure_system.cpp:181-211
* ``interp_2d``    src/internal/measure_system.cpp:213-299

Both are pinned by the reference's known answers in
test/measure_system.cpp:13-92.  Arithmetic is done in float32 where the
reference uses ``float``.
"""
from __future__ import annotations

import math

import numpy as np

INF = float("inf")


def log2_floor(x: int) -> int:
    return 0 if x == 0 else x.bit_length() - 1


def log2_ceil(x: int) -> int:
    l2 = log2_floor(x)
    return l2 + 1 if x & (x - 1) else l2


def interp_time(a, nbytes: int) -> float:
    if not a:
        return INF
    lb, ub = log2_floor(nbytes), log2_ceil(nbytes)
    if ub >= len(a):
        return a[-1] * nbytes / (1 << (len(a) - 1))
    if lb == ub:
        return float(a[lb])
    f32 = np.float32
    num = f32(nbytes - (1 << lb))
    den = f32((1 << ub) - (1 << lb))
    sf = f32(num / den)
    return float(a[lb] * (1 - sf) + a[ub] * sf)


def interp_2d(a, nbytes: int, stride: int) -> float:
    assert stride <= 512
    if not a:
        return INF
    f32 = np.float32
    yi1 = (log2_floor(nbytes) - 6) // 2
    y1 = 1 << (yi1 * 2 + 6)
    yi2 = yi1 if y1 == nbytes else yi1 + 1
    y2 = 1 << (yi2 * 2 + 6)
    xi1 = log2_floor(stride)
    x1 = 1 << xi1
    xi2 = log2_ceil(stride)
    x2 = 1 << xi2
    row = a[min(yi2, len(a) - 1)] if yi2 >= len(a) else a[yi2]
    if xi2 >= len(row):
        xi2 = len(row) - 1
    xi1 = min(xi2, xi1)
    sf_x = f32(0.0) if xi2 == xi1 else f32(f32(stride - x1) / f32(x2 - x1))
    sf_y = f32(0.0) if yi2 == yi1 else f32(f32(nbytes - y1) / f32(y2 - y1))
    if yi2 >= len(a):
        last = a[-1]
        base = f32((1 - sf_x) * f32(last[xi1]) + sf_x * f32(last[xi2]))
        y_max = f32(1 << ((len(a) - 1) * 2 + 6))
        return float(base / y_max * nbytes)
    f1 = f32((1 - sf_x) * f32(a[yi1][xi1]) + sf_x * f32(a[yi1][xi2]))
    f2 = f32((1 - sf_x) * f32(a[yi2][xi1]) + sf_x * f32(a[yi2][xi2]))
    return float(f32((1 - sf_y) * f1 + sf_y * f2))
