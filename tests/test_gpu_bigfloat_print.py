"""BigFloat::print on the GPU (bgpu_bigfloat_to_decimal) against the
reference's own BigFloat::print (src/bigint.cpp:972-1041): identical text for
integer, fractional and mixed values, both signs, default and explicit
fraction lengths, the carry of a fraction that rounds up to 10^d into the
integer part, and large values.

Where the reference's rounding of the scaled fraction is undefined (it lies
in [2^-28, 1/2) and the rounding leaves no digit) the reference is not run and
the device's fraction must print as zeros, which is the value rounding half up
gives there."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import SEED

pytestmark = pytest.mark.gpu
MASK = (1 << 28) - 1


@pytest.fixture(scope="module")
def ref():
    from oracle.pyoracle import Reference, have_reference

    if not have_reference():
        pytest.skip("reference oracle library not built")
    r = Reference()
    if not r.has_bigfloat_print:
        pytest.skip("reference oracle library without ref_bigfloat_print")
    return r


def normal_form(x: int, offset: int):
    """BigFloat(X, offset)'s Digits and point position: X * 2^offset with no
    zero digit at either end."""
    pp = -(offset // 28) if offset < 0 else 0
    v = x << (offset + 28 * pp)
    d = []
    while v:
        d.append(v & MASK)
        v >>= 28
    t = 0
    while d[t] == 0:
        t += 1
    return np.array(d[t:], dtype=np.uint32), pp - t


def default_digits(d, pp) -> int:
    fsize = min(pp, d.size) if pp > 0 else 0
    return math.floor(float(fsize * 28) * math.log10(2))


def digits_int(d) -> int:
    from oracle.pyoracle import digits28_to_limbs

    return int.from_bytes(digits28_to_limbs(d).astype("<u8").tobytes(), "little") if d.size else 0


def undefined(d, pp, dec) -> bool:
    """True when frac * 10^dec lies in [2^-28, 1/2)."""
    if pp <= 0 or dec == 0:
        return False
    frac = digits_int(d[: min(pp, d.size)])
    if not frac:
        return False
    est = frac.bit_length() + dec * math.log2(10)  # log2(frac * 10^dec) within 1
    if est > 28 * pp + 4 or est < 28 * pp - 36:
        return False
    scaled = frac * 10 ** dec
    return (scaled << 28) >= (1 << (28 * pp)) and 2 * scaled < (1 << (28 * pp))


def check(bb, ref, x: int, offset: int, neg: bool, dec: int):
    from oracle.pyoracle import digits28_to_limbs

    d, pp = normal_form(x, offset)
    got = bb.bigfloat_to_decimal(d, pp, neg, dec)
    if undefined(d, pp, dec or default_digits(d, pp)):
        head, frac = got.split(".")
        assert set(frac) == {"0"}, (d.size, pp, dec, got[:40])
        return
    limbs = digits28_to_limbs(from_int_digits(x))
    (din, ppin), want = ref.bigfloat_print(limbs, offset, neg, dec)
    assert np.array_equal(din, d) and ppin == pp
    assert got == want, (d.size, pp, neg, dec, got[:40], want[:40], len(got), len(want))


def from_int_digits(x: int) -> np.ndarray:
    out = []
    while x:
        out.append(x & MASK)
        x >>= 28
    return np.array(out or [0], dtype=np.uint32)


def rand_int(rng, bits: int) -> int:
    nl = (bits + 63) // 64
    v = int.from_bytes(rng.integers(0, 2**64, nl, dtype=np.uint64).tobytes(), "little")
    return (v & ((1 << bits) - 1)) | (1 << (bits - 1))


def test_small_values_all_shapes(bb, ref):
    rng = np.random.default_rng(SEED + 900)
    for trial in range(150):
        x = rand_int(rng, int(rng.integers(1, 300)))
        offset = int(rng.integers(-400, 120))
        dec = [0, 0, 1, 5, 19, 40, 100][trial % 7]
        check(bb, ref, x, offset, bool(trial & 1), dec)


def test_rounding_up_to_the_next_integer(bb, ref):
    """Fractions that round to 10^d: the integer part gains one, with a carry
    through all-ones digits."""
    for int_bits in (0, 1, 28, 100, 280):
        for frac_bits in (40, 60, 200):
            for dec in (1, 3, 10):
                x = ((1 << int_bits) - 1 << frac_bits) | ((1 << frac_bits) - 1)  # int part all ones
                check(bb, ref, x, -frac_bits, False, dec)
                check(bb, ref, x, -frac_bits, True, dec)


def test_integers_and_zero(bb, ref):
    rng = np.random.default_rng(SEED + 901)
    for trial in range(20):
        x = rand_int(rng, int(rng.integers(1, 2000)))
        check(bb, ref, x, int(rng.integers(0, 100)), bool(trial & 1), [0, 7][trial % 2])
    assert bb.bigfloat_to_decimal(np.array([0], np.uint32), 0, False, 0) == "0."
    assert bb.bigfloat_to_decimal(np.array([0], np.uint32), 0, False, 4) == "0.0000"


def test_scaled_fraction_below_one_half(bb, ref):
    """Tiny fractions: below 2^-28 after scaling the reference prints zeros;
    in [2^-28, 1/2) the device prints zeros (the reference is undefined)."""
    for offset in (-30, -35, -40, -57, -90):
        for dec in (1, 2, 8):
            check(bb, ref, 1, offset, False, dec)
            check(bb, ref, (1 << 28) + 1, offset - 28, False, dec)


def test_large_values(bb, ref):
    """2^18- and 2^20-bit values: point inside, above and below the digits."""
    rng = np.random.default_rng(SEED + 902)
    for bits, offset, dec in [(1 << 18, -(1 << 17), 0), (1 << 20, -(1 << 19) - 5, 0), (1 << 18, -(1 << 18) - 100, 0),
                              (1 << 20, -(1 << 20), 1000), (1 << 18, 77, 0)]:
        check(bb, ref, rand_int(rng, bits), offset, False, dec)
