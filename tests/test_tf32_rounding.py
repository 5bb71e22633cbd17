"""The TF32 rounding of the warp-specialised fused Gram's converters (gram_tc.cuh,
tf32_rna_bits): add half the weight of the 13 dropped mantissa bits to the FP32 bit pattern and
clear them.  Checked on the CPU against an independent rounding to 10 explicit mantissa bits,
to nearest with ties away from zero, computed exactly in FP64 from the value itself: random
values over the whole exponent range, exact ties, mantissas that carry into the exponent,
subnormals and zeros, of both signs.  (The GPU tests compare the kernel's Gram bit for bit with
the kernel that rounds with cvt.rna.tf32.f32, on blocks of a single k-tile.)"""
import numpy as np


def _trick(x32):
    b = x32.view(np.uint32).astype(np.uint64)
    r = ((b + 0x1000) & 0xFFFFE000).astype(np.uint32)
    return r.view(np.float32)


def _exact_rna(x32):
    """Round |x| to a multiple of its TF32 ulp (2^(e - 10) for a normal of exponent e; the
    subnormal spacing 2^-149 times 2^13 below 2^-126), ties away from zero, in FP64 (exact:
    every FP32 value and every such multiple is an FP64 number)."""
    x = x32.astype(np.float64)
    a = np.abs(x)
    out = np.zeros_like(a)
    nz = a > 0
    e = np.floor(np.log2(a[nz]))
    # log2 can land one off at exact powers of two: fix e so that 2^e <= a < 2^(e+1)
    e = np.where(2.0 ** e > a[nz], e - 1, e)
    e = np.where(2.0 ** (e + 1) <= a[nz], e + 1, e)
    ulp = np.where(e < -126, 2.0 ** (-149 + 13), 2.0 ** (e - 10))
    q = a[nz] / ulp                      # exact: a power-of-two division
    out[nz] = np.floor(q + 0.5) * ulp    # q + 0.5 is exact (q < 2^24)
    return np.copysign(out, x).astype(np.float32)


def _check(x32):
    got, want = _trick(x32), _exact_rna(x32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (
        x32[got.view(np.uint32) != want.view(np.uint32)][:5])


def test_random_values_over_the_exponent_range():
    rng = np.random.default_rng(20240611)
    bits = rng.integers(0, 0x7F7FFFFF, size=400_000, dtype=np.uint64).astype(np.uint32)
    x = bits.view(np.float32)
    x = x[np.abs(x) < 3.0e38]  # keep the rounded value finite
    _check(x)
    _check(-x)


def test_ties_carries_subnormals_and_zeros():
    mant = np.array([0x000000, 0x000FFF, 0x001000, 0x001001, 0x002FFF, 0x003000, 0x7FEFFF, 0x7FF000, 0x7FFFFF],
                    dtype=np.uint32)
    exps = np.array([0, 1, 2, 100, 127, 128, 200, 253], dtype=np.uint32)
    bits = (exps[:, None] << 23 | mant[None, :]).ravel()
    x = bits.view(np.float32)
    _check(x)
    _check(-x)
    # exact ties round away from zero: 1 + 2^-11 -> 1 + 2^-10; carry into the exponent at 2 - 2^-12
    assert _trick(np.array([1.0 + 2.0 ** -11], np.float32))[0] == np.float32(1.0 + 2.0 ** -10)
    assert _trick(np.array([2.0 - 2.0 ** -12], np.float32))[0] == np.float32(2.0)
    assert _trick(np.array([-(1.0 + 2.0 ** -11)], np.float32))[0] == np.float32(-(1.0 + 2.0 ** -10))
    assert _trick(np.array([0.0], np.float32)).view(np.uint32)[0] == 0
    assert _trick(np.array([-0.0], np.float32)).view(np.uint32)[0] == 0x80000000


def test_lo_part_is_the_exact_residual_and_rounds_again():
    """hi = rna(x), lo = rna(x - hi): x - hi is exact in FP32 (hi is within half a TF32 ulp of x),
    and hi + lo carries x to 2^-22 of |x|."""
    rng = np.random.default_rng(7)
    x = (rng.standard_normal(100_000) * 10.0 ** rng.uniform(-20, 20, 100_000)).astype(np.float32)
    hi = _trick(x)
    res = (x.astype(np.float64) - hi.astype(np.float64))
    assert np.array_equal(res.astype(np.float32).astype(np.float64), res)  # exact in FP32
    lo = _trick(res.astype(np.float32))
    err = np.abs(x.astype(np.float64) - hi.astype(np.float64) - lo.astype(np.float64))
    assert np.all(err <= 2.0 ** -22 * np.abs(x.astype(np.float64)))
