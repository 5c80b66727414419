"""The digit-split (ozaki) contraction of the fused stage, restated in numpy on
the CPU: six signed 7-bit digits per value at a power-of-two scale shared by a
row (data) or a column (table), the 21 digit pairs with i + j <= 5 summed by
weight group exactly in integers (as the int32 TMEM accumulators of
tcgen05.mma kind::i8 sum them), combined in FP64.  Checks the digit range
and the exactness of the decomposition, that every group sum fits int32 with
a wide margin, and that the synthesis- and analysis-shaped Legendre
contractions of the l_max = 255 grid are accurate to ~1e-12 of their scale
(the FP64 oracle tables and the benchmark's spectral decay)."""

import numpy as np
import pytest

from oracle import grid as og

D, G = 6, 6  # digits per operand, weight groups kept (i + j <= 5)


OFFSET = 64 * sum(1 << (7 * (5 - i)) for i in range(D))  # 64 sum_i 2^(7 (5 - i))


def digits(x, axis):
    """(digit planes, exponents) as the pack kernels form them: Y = rint(x 2^(41 - e))
    (|Y| <= 2^41), written in balanced base 128 through the independent shifts of
    Y + OFFSET (each base-128 digit minus 64), so x = 2^(e - 6) sum_i d_i 2^(-7 i)
    to 2^(e - 42); e per row (axis = 1) or column (axis = 0), |x| < 2^e."""
    mx = np.abs(x).max(axis=axis, keepdims=True)
    e = np.where(mx > 0, np.frexp(mx)[1], 0)
    Y = np.rint(np.ldexp(x, 41 - e)).astype(np.int64)
    U = Y + OFFSET
    ds = [(U >> 35) - 64] + [((U >> (7 * (5 - i))) & 127) - 64 for i in range(1, D)]
    return ds, e


def _pow2(k):
    import struct

    return struct.unpack("<d", struct.pack("<q", (k + 1023) << 52))[0]


def oz_scale(v, s):
    """v 2^s as the epilogues compute it (s <= 1023), for Python floats."""
    if s >= -1022:
        return v * _pow2(s)
    return (v * _pow2(max(s + 1022, -1022))) * 2.0 ** -1022


def oz_scale_up(v, s):
    """v 2^s as the packs compute it (s >= -1022)."""
    if s <= 1023:
        return v * _pow2(s)
    return (v * _pow2(min(s - 1023, 1023))) * 2.0 ** 1023


def test_scaling_rounds_like_ldexp():
    """The kernels' power-of-two scaling equals ldexp (one rounding) over the
    exponents they use: digit extraction of values down to the subnormals, and
    the epilogue's integer sums below 2^59 scaled into the subnormal range."""
    import math
    import random

    rnd = random.Random(0)
    for _ in range(100000):
        e = rnd.randint(-1073, 1023)
        v = rnd.uniform(-1.0, 1.0) * 2.0 ** e
        if v != 0.0:
            s = 41 - math.frexp(v)[1]
            assert oz_scale_up(v, s) == math.ldexp(v, s)
        w, t = float(rnd.randint(-2 ** 59, 2 ** 59)), rnd.randint(-2200, 60)
        assert oz_scale(w, t) == math.ldexp(w, t)


def digit_bytes(v, e):
    """The pack kernels' byte form of the digits of v (scale 2^e), restated with
    exact rationals: T = fma(v, 2^(41 - e), 1.5 2^52 + OFFSET) rounded once to
    the nearest double (ties to even), the mantissa of T = 2^51 + U split into
    its low and high words, the six 7-bit fields read with 32-bit shifts
    (d_0 from eight bits of the high word, the rest by a borrow-free per-byte
    subtraction of 64)."""
    from fractions import Fraction

    x = Fraction(v) * Fraction(2) ** (41 - e) + int(1.5 * 2 ** 52) + OFFSET
    n, r = divmod(x, 1)
    n = int(n)
    if r > Fraction(1, 2) or (r == Fraction(1, 2) and n % 2):
        n += 1
    assert 2 ** 52 <= n < 2 ** 53  # one binade: the ulp of T is 1
    mant = n - 2 ** 52
    lo, hi = mant & 0xFFFFFFFF, (0x433 << 20) | (mant >> 32)
    raw = [((hi << 32 | lo) >> 28) & 127, (lo >> 21) & 127, (lo >> 14) & 127, (lo >> 7) & 127,
           lo & 127]
    bias = lambda w: (((w | 0x80) - 0x40) ^ 0x80) & 0xFF  # one byte of oz_bias_bytes
    return [((hi >> 3) + 192) & 0xFF] + [bias(w) for w in raw]


def test_byte_digits_equal_integer_digits():
    """The fma / word-split digits of the pack kernels equal the integer
    method's digits (as int8 bytes) for values across the exponent range,
    including the rounding ties and |v| rounding up to 2^e (d_0 = 64)."""
    import math
    import random

    rnd = random.Random(1)
    cases = []
    for _ in range(4000):
        e = rnd.randint(-900, 900)
        v = rnd.uniform(-1.0, 1.0) * 2.0 ** e
        cases.append((v, math.frexp(v)[1] if v else 0))
        cases.append((v, (math.frexp(v)[1] if v else 0) + rnd.randint(0, 12)))  # row scale above
    for e in (0, 5, -3):
        top = 2.0 ** e
        cases += [(math.nextafter(top, 0.0), e), (-math.nextafter(top, 0.0), e)]  # round to 2^41
        cases += [((k + 0.5) * 2.0 ** (e - 41), e) for k in (-4, -3, 0, 1, 2, 7)]  # exact ties
    cases += [(0.0, 0), (0.0, 7), (5e-324, -1073), (-5e-324, -1073)]
    for v, e in cases:
        Y = int(np.rint(np.ldexp(v, 41 - e)))
        assert abs(Y) <= 2 ** 41
        U = Y + OFFSET
        ref = [(U >> 35) - 64] + [((U >> (7 * (5 - i))) & 127) - 64 for i in range(1, D)]
        assert digit_bytes(v, e) == [d & 0xFF for d in ref], (v, e)


def contract(A, B):
    da, ea = digits(A, 1)
    db, eb = digits(B, 0)
    out = np.zeros((A.shape[0], B.shape[1]))
    groups = []
    for g in range(G):
        C = np.zeros(out.shape, dtype=np.int64)
        for i in range(g + 1):
            C += da[i] @ db[g - i]  # exact integer sums, as the int32 accumulators
        groups.append(C)
    for g in range(G - 1, -1, -1):
        out = out / 128.0 + groups[g]
    return np.ldexp(out, ea + eb - 12), groups, (da, db)


def test_digits_are_small_and_reconstruct():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((8, 300)) * np.exp(rng.uniform(-30, 30, (8, 1)))
    ds, e = digits(x, 1)
    for d in ds:
        assert np.abs(d).max() <= 64
    back = sum(np.ldexp(d.astype(np.float64), -7 * i) for i, d in enumerate(ds))
    err = np.abs(np.ldexp(back, e - 6) - x) / np.ldexp(1.0, e)
    assert err.max() <= 2.0 ** -41


@pytest.mark.parametrize("kind", ["synthesis", "analysis"])
def test_contraction_accuracy_at_lmax_255(kind):
    g = og.Grid(255)
    rng = np.random.default_rng(1)
    worst, lim = 0.0, 0
    for m in (0, 17, 64, 128, 200, 250):
        rows = np.nonzero(g.lm2m == m)[0]
        l = g.lm2l[rows]
        if kind == "synthesis":
            # rows: scaled spectra over l (the row programs' l(l+1) included)
            A = rng.standard_normal((16, len(rows))) * (1e-4 * (l + 1.0) ** -2 * l * (l + 1))
            B = g.Plm[rows]
        else:
            # rows: weighted Fourier rows of a vector product over theta (1/sin^2)
            th = g.theta_ord[:g.NHS]
            c = rng.standard_normal((16, len(rows))) * (1e-4 * (l + 1.0) ** -2)
            A = (c @ g.dPlm[rows]) * (g.gauss[:g.NHS] / np.sin(th) ** 2)
            B = g.Plm[rows].T
        ref = A @ B
        got, groups, _ = contract(A, B)
        worst = max(worst, np.abs(got - ref).max() / np.abs(ref).max())
        lim = max(lim, max(int(np.abs(c).max()) for c in groups))
    assert worst < 2e-11, worst
    assert lim < 2 ** 28  # int32 accumulators with >= 8 bits of margin at this K
