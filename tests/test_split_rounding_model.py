"""Error model of the hi/lo operand split of the tcgen05 forms, restated in
numpy (no GPU).

Every split kernel rounds an FP64 value x once to FP32, f = fp32(x), then
takes hi = rn16(f) and lo = rn16(f - hi).  These tests pin the two facts the
tolerances of the split-form parity tests rest on:

- f - hi is exact in FP32, so lo is the correctly rounded residual of f;
- with u = 2^-11 (fp16) or 2^-8 (bf16), hi + lo represents x to
  u^2 + 2^-24 relative (1.25 * 2^-22 for fp16, operands scaled into
  [2^14, 2^15)), and the three-product form hi*hi' + hi*lo' + lo*hi' of x*y
  is good to 3 u^2 + 2 * 2^-24 of |x||y|: the dropped lo*lo' and the two
  representation errors.
"""
import numpy as np


def _bf16(a32):
    """Round-to-nearest-even of float32 values to bfloat16, returned as float32."""
    u = np.asarray(a32, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def _split(x, fp16):
    f = x.astype(np.float32)
    if fp16:
        hi = f.astype(np.float16).astype(np.float32)
        res = f - hi
        lo = res.astype(np.float16).astype(np.float32)
    else:
        hi = _bf16(f)
        res = f - hi
        lo = _bf16(res)
    return f, hi, res, lo


def _scaled_operand(rng, n):
    """Entries of mixed magnitude, scaled by a power of two so that the
    largest lies in [2^14, 2^15), as the fp16 split scales its operands."""
    x = rng.standard_normal(n) * np.exp(rng.uniform(-6.0, 0.0, n))
    s = 2.0 ** np.floor(np.log2(32768.0 / np.abs(x).max()))
    return x * s


def test_residual_is_exact_in_fp32():
    rng = np.random.default_rng(0)
    for fp16 in (True, False):
        x = _scaled_operand(rng, 200_000) if fp16 else rng.standard_normal(200_000)
        f, hi, res, _ = _split(x, fp16)
        exact = f.astype(np.float64) - hi.astype(np.float64)
        assert np.array_equal(res.astype(np.float64), exact)


def test_representation_error_bound_fp16():
    rng = np.random.default_rng(1)
    x = _scaled_operand(rng, 400_000)
    _, hi, _, lo = _split(x, True)
    rep = hi.astype(np.float64) + lo.astype(np.float64)
    # Relative to the element the bound is 2^-22 (lo) + 2^-24 (fp32 of x) for
    # |x| >= 2^-3, where even a subnormal lo (absolute error <= 2^-25) stays
    # within 2^-22 |x|.
    big = np.abs(x) >= 2.0 ** -3
    rel = np.abs(rep[big] - x[big]) / np.abs(x[big])
    assert rel.max() <= 1.2501 * 2.0 ** -22
    # Relative to the operand's largest entry it holds everywhere.
    assert np.abs(rep - x).max() <= 1.2501 * 2.0 ** -22 * np.abs(x).max()


def test_three_product_error_model():
    rng = np.random.default_rng(2)
    for fp16, u in ((True, 2.0 ** -11), (False, 2.0 ** -8)):
        bound = (3.0 * u * u + 2.0 * 2.0 ** -24) * (1.0 + 4.0 * u)
        x = _scaled_operand(rng, 100_000) if fp16 else rng.standard_normal(100_000)
        y = _scaled_operand(rng, 100_000) if fp16 else rng.standard_normal(100_000)
        _, xh, _, xl = _split(x, fp16)
        _, yh, _, yl = _split(y, fp16)
        xh, xl, yh, yl = (a.astype(np.float64) for a in (xh, xl, yh, yl))
        prod = xh * yh + xh * yl + xl * yh
        err = np.abs(prod - x * y) / (np.abs(x) * np.abs(y))
        # fp16: |x|, |y| >= 2^-3, as above.
        keep = (np.abs(x) >= 2.0 ** -3) & (np.abs(y) >= 2.0 ** -3) if fp16 else np.ones(err.shape, bool)
        assert err[keep].max() <= bound
