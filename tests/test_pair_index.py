"""The closed-form inversion of the triangular pair index used by the
geometric modes of the triangle and 4-clique kernels (gr_tri.cu, gr_quad.cu):
pair t of the k(k-1)/2 pairs (x, y), x < y < k, in row-major order has
x = floor((2k - 1 - sqrt((2k - 1)^2 - 8t)) / 2) in single precision, then one
step up or down against the exact integer row starts, and
y = t - x(2k - 1 - x)/2 + x + 1.  The kernels rely on it being a bijection for
every row length up to 1024 (the capacity of the long-row launch), also with
a square root a few ulp off.  Up to 256 members the kernels use no
adjustment: 2.5e-4 is added to the single-precision estimate before it is
truncated (pair_row_biased in gr_internal.cuh), which must give the exact
row for every pair with the root 3 ulp off either way."""
import numpy as np
import pytest


def _invert(k, t, sqrt_err_ulp=0):
    f32 = np.float32
    k2m1 = 2 * k - 1
    disc = f32(k2m1 * k2m1) - f32(8.0) * t.astype(f32)
    sq = np.sqrt(np.maximum(disc, f32(0))).astype(f32)
    if sqrt_err_ulp:
        sq = (sq * f32(1 + sqrt_err_ulp * 2.0 ** -23)).astype(f32)
    x = np.trunc((f32(0.5) * (f32(k2m1) - sq)).astype(f32)).astype(np.int64)
    x = np.clip(x, 0, k - 2)
    x = x + ((x + 1) * (k2m1 - x - 1) // 2 <= t)
    x = x - (x * (k2m1 - x) // 2 > t)
    y = t - x * (k2m1 - x) // 2 + x + 1
    return x, y


@pytest.mark.parametrize("err", [-3, 0, 3])
def test_pair_index_inversion_is_a_bijection(err):
    for k in range(2, 1025):
        npair = k * (k - 1) // 2
        assert (2 * k - 1) ** 2 < 2 ** 24 and 8 * npair < 2 ** 24  # exact in float32
        t = np.arange(npair, dtype=np.int64)
        x, y = _invert(k, t, err)
        assert np.all((0 <= x) & (x < y) & (y < k)), k
        # row-major order back from (x, y) gives t again
        assert np.array_equal(x * (2 * k - 1 - x) // 2 + (y - x - 1), t), k


def _invert_biased(k, t, sqrt_err_ulp=0):
    """The kernels' form: biased estimate, adjusted only beyond 256 members."""
    f32 = np.float32
    k2m1 = 2 * k - 1
    disc = f32(k2m1 * k2m1) - f32(8.0) * t.astype(f32)
    sq = np.sqrt(np.maximum(disc, f32(0))).astype(f32)
    if sqrt_err_ulp:
        sq = (sq * f32(1 + sqrt_err_ulp * 2.0 ** -23)).astype(f32)
    u = (f32(0.5) * (f32(k2m1) - sq)).astype(f32)
    x = np.trunc((u + f32(2.5e-4)).astype(f32)).astype(np.int64)
    if k > 256:
        x = np.clip(x, 0, k - 2)
        x = x + ((x + 1) * (k2m1 - x - 1) // 2 <= t)
        x = x - (x * (k2m1 - x) // 2 > t)
    y = t - x * (k2m1 - x) // 2 + x + 1
    return x, y


@pytest.mark.parametrize("err", [-3, 0, 3])
def test_biased_row_is_exact_without_adjustment(err):
    # every k of the unadjusted form, and the adjusted form just above it and
    # at the long-row capacity
    for k in list(range(2, 301)) + list(range(1000, 1025)):
        npair = k * (k - 1) // 2
        t = np.arange(npair, dtype=np.int64)
        x, y = _invert_biased(k, t, err)
        assert np.all((0 <= x) & (x < y) & (y < k)), k
        assert np.array_equal(x * (2 * k - 1 - x) // 2 + (y - x - 1), t), k
        if k <= 256:
            # exact before any adjustment
            k2m1 = 2 * k - 1
            exact = np.floor((k2m1 - np.sqrt(float(k2m1 * k2m1) - 8.0 * t)) / 2).astype(np.int64)
            assert np.array_equal(x, exact), k
