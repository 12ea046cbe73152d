"""The split-precision products of the tensor-core kernels, restated in
numpy: every operand x in a head and a tail, hi = round(x), lo = round(x -
hi), and sum a*c ~ sum (a_hi c_hi + a_lo c_hi + a_hi c_lo) with the products
exact.  The roundings are the kernels' own integer-pipe forms (TF32: the
magnitude to 10 mantissa bits, ties away; BF16: nearest, ties to even).

Bounds checked, relative to sum |a c|: 3xTF32 drops a_lo c_lo and the tails'
rounding, about 3 * 2^-22 per term (bar 1e-6); BF16x3, about 3 * 2^-16 (bar
1e-4).  K = 10 (the gather's sums over y, the three products folded along
K as A = [a_hi | a_lo | a_hi], B = [c_hi | c_hi | c_lo]) and K = 130 (the
mode products)."""
import numpy as np
import pytest


def tf32_rna(x):
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x1000) & 0xFFFFE000).astype(np.uint32).view(np.float32)


def bf16_rne(x):
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32).view(np.float32)


def split(x, rnd):
    x = np.asarray(x, dtype=np.float32)
    hi = rnd(x)
    lo = rnd((x - hi).astype(np.float32))
    return hi, lo


def folded(a, c, rnd):
    """The gather's K-folded operands: A = [a_hi | a_lo | a_hi], B = [c_hi | c_hi | c_lo]."""
    ah, al = split(a, rnd)
    ch, cl = split(c, rnd)
    A = np.concatenate([ah, al, ah], axis=-1).astype(np.float64)
    B = np.concatenate([ch, ch, cl], axis=-1).astype(np.float64)
    return (A * B).sum(axis=-1)


@pytest.mark.parametrize("rnd, bar", [(tf32_rna, 1e-6), (bf16_rne, 1e-4)], ids=["3xtf32", "bf16x3"])
@pytest.mark.parametrize("k", [10, 130])
def test_split_products_bound(rnd, bar, k):
    rng = np.random.default_rng(k)
    # values of alternating sign and a few decades of magnitude, like the
    # stencil coefficients and the smoothing tables
    a = (rng.standard_normal((2000, k)) * np.exp(rng.uniform(-3, 3, (2000, k)))).astype(np.float32)
    c = (rng.standard_normal((2000, k)) * np.exp(rng.uniform(-3, 3, (2000, k)))).astype(np.float32)
    exact = (a.astype(np.float64) * c.astype(np.float64)).sum(axis=1)
    scale = np.abs(a.astype(np.float64) * c.astype(np.float64)).sum(axis=1)
    err = np.abs(folded(a, c, rnd) - exact) / scale
    assert err.max() < bar, err.max()
    # the two-term form (a_hi c_hi alone) is far worse: the tails matter
    ah, _ = split(a, rnd)
    ch, _ = split(c, rnd)
    one = (ah.astype(np.float64) * ch.astype(np.float64)).sum(axis=1)
    assert (np.abs(one - exact) / scale).max() > 10 * bar


def test_heads_are_representable():
    rng = np.random.default_rng(3)
    x = rng.standard_normal(10000).astype(np.float32)
    hi, lo = split(x, tf32_rna)
    assert np.all(hi.view(np.uint32) & 0x1FFF == 0) and np.all(lo.view(np.uint32) & 0x1FFF == 0)
    bh, bl = split(x, bf16_rne)
    assert np.all(bh.view(np.uint32) & 0xFFFF == 0) and np.all(bl.view(np.uint32) & 0xFFFF == 0)
    # hi + lo reproduces x to 2^-22 (TF32) and 2^-16 (BF16) of |x|
    assert np.max(np.abs((hi.astype(np.float64) + lo) - x) / np.abs(x)) < 2 ** -21
    assert np.max(np.abs((bh.astype(np.float64) + bl) - x) / np.abs(x)) < 2 ** -15
