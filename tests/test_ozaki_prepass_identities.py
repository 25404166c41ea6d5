"""Integer identities the Ozaki pre-pass kernels rely on (CPU only).

The digit-slicing kernel (ozaki_slice_kernel in rblas_b200/csrc/gemm_umma.cu)
balances the base-256 digits of Y = floor(x * 2^n) with a byte-wise bias and
flip instead of the low-to-high carry loop, and packs four elements' digit t
into one word with byte permutes. The row-exponent kernels take frexp_exp of
the largest |x| bit pattern instead of the largest frexp_exp. Each form must
give exactly what the slower one gives; these tests restate both in Python
and compare them on seeded random and boundary values."""
from __future__ import annotations

import math
import random
import struct

import pytest


def _digits_carry_loop(Y: int, S: int) -> list[int]:
    """Signed top digit and unsigned lower digits of Y, balanced from the least
    significant up: a digit >= 128 becomes digit - 256 with a carry of 1."""
    d = [(Y >> (8 * (S - 1))) if t == 0 else (Y >> (8 * (S - 1 - t))) & 0xFF for t in range(S)]
    for t in range(S - 1, 0, -1):
        if d[t] >= 128:
            d[t] -= 256
            d[t - 1] += 1
    return [v & 0xFF for v in d]


def _digits_bias_flip(Y: int, S: int) -> list[int]:
    """Digit t is byte S-1-t of Z = (Y + B) ^ B, B = 0x80 in each of the S-1 low bytes."""
    B = 0x0080808080808080 >> (8 * (8 - S))
    Z = ((Y + B) & (2**64 - 1)) ^ B
    return [(Z >> (8 * (S - 1 - t))) & 0xFF for t in range(S)]


def _byte_perm(x: int, y: int, sel: int) -> int:
    """__byte_perm(x, y, sel): result byte k is byte sel[k] of the 8-byte pool y:x."""
    pool = [(x >> (8 * i)) & 0xFF for i in range(4)] + [(y >> (8 * i)) & 0xFF for i in range(4)]
    return sum(pool[(sel >> (4 * k)) & 0x7] << (8 * k) for k in range(4))


@pytest.mark.parametrize("S", range(2, 9))
def test_bias_flip_digits_equal_carry_loop(S):
    rng = random.Random(100 + S)
    lim = 1 << (7 + 8 * (S - 1) - 1)  # |Y| < 2^(N-1), N = 7 + 8(S-1)
    cases = [0, 1, -1, lim - 1, -lim, 127, 128, -128, 255, 256, -129, -256]
    cases += [rng.randrange(-lim, lim) for _ in range(20000)]
    for t in range(1, S):  # lower digits on the balancing boundaries
        sh = 8 * (S - 1 - t)
        for v in (0x00, 0x7F, 0x80, 0xFF):
            for _ in range(50):
                cases.append((rng.randrange(-lim, lim) & ~(0xFF << sh)) | (v << sh))
    for Y in cases:
        if -lim <= Y < lim:
            assert _digits_bias_flip(Y, S) == _digits_carry_loop(Y, S), (S, Y)


@pytest.mark.parametrize("S", range(2, 9))
def test_byte_permute_packing(S):
    """Word g of plane t holds digit t of elements 4g .. 4g+3, lowest byte first."""
    rng = random.Random(200 + S)
    B = 0x0080808080808080 >> (8 * (8 - S))
    lim = 1 << (7 + 8 * (S - 1) - 1)
    for _ in range(500):
        Z = [((rng.randrange(-lim, lim) + B) & (2**64 - 1)) ^ B for _ in range(4)]
        lo = [z & 0xFFFFFFFF for z in Z]
        hi = [z >> 32 for z in Z]
        for t in range(S):
            b = S - 1 - t
            src = lo if b < 4 else hi
            sel = (b & 3) | (((b & 3) + 4) << 4)
            word = _byte_perm(_byte_perm(src[0], src[1], sel), _byte_perm(src[2], src[3], sel), 0x5410)
            assert word == sum(((Z[q] >> (8 * b)) & 0xFF) << (8 * q) for q in range(4))


def _bits(x: float) -> int:
    return struct.unpack("<q", struct.pack("<d", x))[0]


def _from_bits(b: int) -> float:
    return struct.unpack("<d", struct.pack("<q", b))[0]


def _frexp_exp(x: float) -> int:
    """The kernels' exponent: e with |x| in [2^(e-1), 2^e) for finite nonzero x
    (frexp), field - 1022 = 1025 for inf and NaN."""
    f = (_bits(x) >> 52) & 0x7FF
    return f - 1022 if f != 0 else math.frexp(x)[1]


def test_row_exponent_from_largest_abs_bits():
    rng = random.Random(7)
    specials = [0.0, -0.0, 5e-324, -5e-324, 2.2250738585072014e-308, 2.225073858507201e-308, 1.0, -1.0,
                1.7976931348623157e308, float("inf"), float("-inf"), float("nan")]
    for trial in range(3000):
        n = rng.randrange(1, 40)
        row = []
        for _ in range(n):
            kind = rng.random()
            if kind < 0.1:
                row.append(rng.choice(specials))
            elif kind < 0.2:
                row.append(rng.uniform(-1, 1) * 2.0 ** -1070)  # subnormal
            else:
                row.append(math.ldexp(rng.uniform(-1, 1), rng.randrange(-1021, 1023)))
        nonzero = [v for v in row if v != 0.0]
        want = max(_frexp_exp(v) for v in nonzero) if nonzero else None
        best = max(_bits(v) & 0x7FFFFFFFFFFFFFFF for v in row)
        got = _frexp_exp(_from_bits(best)) if best != 0 else None
        assert got == want, row
