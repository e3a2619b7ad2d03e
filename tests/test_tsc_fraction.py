"""The TSC fraction of a fixed-point coordinate, as the deposit and the
gradient interpolation compute it (axis_of in lageunha_b200/csrc/pm.cu).

The reference forms x - near in double (Cosmos/pmmain.h:86-120 with XYZDBL
positions); the engine has the 32-bit fraction fr of u * n and needs the
float of fr 2^-32 (or fr 2^-32 - 1 past the midpoint). Both are a 32-bit
integer times 2^-32, so rounding the integer to float (round to nearest
even) and scaling by the power of two gives the same bits as rounding the
exact double: the kernels use FP32 only. Checked here bit for bit on random
fractions and the edge values.
"""
import numpy as np


def _fp64_form(fr):
    hi = fr > 0x80000000
    return np.where(hi, fr.astype(np.float64) * 2.0 ** -32 - 1.0, fr.astype(np.float64) * 2.0 ** -32).astype(np.float32)


def _fp32_form(fr):
    hi = fr > 0x80000000
    neg = (np.uint64(2 ** 32) - fr) % np.uint64(2 ** 32)
    scale = np.float32(2.0 ** -32)
    return np.where(hi, -(neg.astype(np.float32) * scale), fr.astype(np.float32) * scale).astype(np.float32)


def test_fraction_bits_match_the_fp64_form():
    rng = np.random.default_rng(3)
    edges = np.array([0, 1, 2, 2 ** 24 - 1, 2 ** 24, 2 ** 24 + 1, 2 ** 31 - 1, 2 ** 31, 2 ** 31 + 1,
                      2 ** 32 - 2 ** 8 - 1, 2 ** 32 - 2, 2 ** 32 - 1], dtype=np.uint64)
    fr = np.concatenate([rng.integers(0, 2 ** 32, 1_000_000, dtype=np.uint64), edges])
    a, b = _fp64_form(fr), _fp32_form(fr)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_scale_constant_is_exactly_two_to_minus_32():
    assert float(np.float32(2.3283064365386963e-10)) == 2.0 ** -32
