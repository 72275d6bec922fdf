"""The cell index's division-free fast path, restated in float32 numpy.

The kernels compute the reference's cell index trunc((x - lo) / (hi - lo) * g), clamped
to [0, g - 1] (src/find_neighbors_kernel.cu:11-22), as floor((x - lo) * inv * g) with
inv = 1 / (hi - lo) rounded to float, except where that product lies within
(g + 1) * 2^-20 of an integer (or is NaN), where they divide. This checks the argument
that the two agree, with the same IEEE float32 operations, on tens of millions of
positions in and around boxes of the workloads' sizes, boundary neighbourhoods
included.
"""
from __future__ import annotations

import numpy as np
import pytest

f32 = np.float32


def exact(x, lo, hi, g):
    t = ((x - f32(lo)) / (f32(hi) - f32(lo))) * f32(g)
    with np.errstate(invalid="ignore"):
        k = np.where(np.isnan(t), 0, np.trunc(np.clip(t, -2.0**31, 2.0**31 - 1))).astype(np.int64)
    return np.clip(k, 0, g - 1)


def fast(x, lo, hi, g):
    length = f32(f32(hi) - f32(lo))
    inv = f32(1.0 / float(length))
    err = f32(np.ldexp(float(g) + 1.0, -20))
    t = ((x - f32(lo)) * inv) * f32(g)
    k = np.floor(t)
    with np.errstate(invalid="ignore"):
        fr = t - k
    inside = (t >= f32(-0.5)) & (t < f32(g) + f32(0.5))
    safe = inside & (fr >= err) & (fr <= f32(1) - err)
    out = np.where(t < f32(-0.5), 0, np.where(t >= f32(g) + f32(0.5), g - 1, -1)).astype(np.int64)
    kk = np.nan_to_num(k, nan=0.0, posinf=0.0, neginf=0.0).astype(np.int64)
    out = np.where(safe, np.clip(kk, 0, g - 1), out)
    slow = out < 0
    out[slow] = exact(x[slow], lo, hi, g)
    return out, float(slow.mean())


BOXES = [(-0.5, 0.5, 181), (0.0, 0.5, 90), (-1.5874010519681994, 1.5874010519681994, 453),
         (0.0, 1.5875, 226), (-1.0, 1.0, 288), (0.0, 1.0, 144), (-0.05, 0.05, 14),
         (-1.0, 1.0, 1), (0.0, 0.1, 1)]


@pytest.mark.parametrize("lo,hi,g", BOXES)
def test_fast_cell_index_equals_reference_expression(lo, hi, g):
    rng = np.random.default_rng(g)
    L = hi - lo
    x = rng.uniform(lo - 0.2 * L, hi + 0.2 * L, 4_000_000).astype(f32)
    _, slow = fast(x, lo, hi, g)
    assert slow < 4 * (g + 1) * 2.0**-20 + 1e-4      # the division is rare
    # positions next to every cell boundary, a few ulps either side
    b = (f32(lo) + (np.arange(g + 1, dtype=np.float64) * L / g)).astype(f32)
    near = np.concatenate([np.nextafter(b, f32(np.inf) * s).astype(f32) for s in (1, -1)] + [b])
    for _ in range(4):
        near = np.concatenate([near, np.nextafter(near, f32(np.inf)), np.nextafter(near, f32(-np.inf))])
    x = np.concatenate([x, near, np.array([np.nan, np.inf, -np.inf], f32)])
    got, _ = fast(x, lo, hi, g)
    np.testing.assert_array_equal(got, exact(x, lo, hi, g))
