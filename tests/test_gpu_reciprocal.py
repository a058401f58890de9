"""Device-resident BigFloat::reciprocal (bgpu_reciprocal_digits) against the
reference's own BigFloat::reciprocal (src/bigint.cpp:1044-1071) on the same
BigFloat: digits, point position and sign identical."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED, rand_limbs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    from oracle.pyoracle import Reference, have_reference

    if not have_reference():
        pytest.skip("reference oracle library not built")
    r = Reference()
    if not r.has_bigfloat_reciprocal:
        pytest.skip("reference oracle library without ref_bigfloat_reciprocal")
    return r


def check(bb, ref, limbs, offset, neg, precision):
    (din, ppin, nin), (want, wpp, wneg) = ref.bigfloat_reciprocal(limbs, offset, neg, precision)
    got, pp, ng = bb.reciprocal_digits(din, ppin, nin, precision)
    assert pp == wpp and ng == wneg, (limbs.size, offset, neg, precision, pp, wpp)
    assert np.array_equal(got, want), (limbs.size, offset, neg, precision, got.size, want.size)


def test_small_values_all_precisions(bb, ref):
    """Short values, every precision from 0 to 40 digits, both signs, points
    left and right of the digits."""
    rng = np.random.default_rng(SEED + 400)
    for trial in range(60):
        limbs = rand_limbs(rng, int(rng.integers(1, 4)))
        check(bb, ref, limbs, int(rng.integers(-200, 200)), bool(trial & 1), trial % 41)


def test_powers_of_two_and_all_ones(bb, ref):
    """b = 1/2 exactly makes 1 - b x vanish (the zero branches of mul and
    add_or_sub); all-ones limbs make long borrow chains."""
    for k in (0, 1, 27, 28, 29, 63, 64, 200, 5000):
        limbs = np.zeros(k // 64 + 1, dtype=np.uint64)
        limbs[-1] = np.uint64(1 << (k % 64))
        for prec in (0, 1, 5, 64):
            check(bb, ref, limbs, -k // 2, k % 3 == 0, prec)
    for n in (1, 3, 100, 2000):
        check(bb, ref, np.full(n, np.uint64(0xFFFFFFFFFFFFFFFF)), 0, False, 0)
        check(bb, ref, np.full(n, np.uint64(0xFFFFFFFFFFFFFFFF)), 17, True, 3 * n)


@pytest.mark.parametrize("bits,prec", [(1 << 12, 0), (1 << 16, 0), (1 << 16, 10000), (1 << 18, 0),
                                       (1 << 20, 0), (1 << 20, 2000), (1 << 22, 0)])
def test_sizes_through_the_methods(bb, ref, bits, prec):
    """Precisions whose products run on schoolbook, Karatsuba and the NTT
    (the last iterations of a 2^22-bit reciprocal are 2^22-bit products)."""
    rng = np.random.default_rng(SEED + 401 + bits.bit_length())
    check(bb, ref, rand_limbs(rng, bits // 64), -(bits // 3), False, prec)


def test_errors(bb):
    with pytest.raises(bb.BigIntGPUError) as e:
        bb.reciprocal_digits(np.array([0], dtype=np.uint32))  # division by zero
    assert e.value.code == -1
    with pytest.raises(bb.BigIntGPUError):
        bb.reciprocal_digits(np.array([5, 0], dtype=np.uint32))  # leading zero digit
    with pytest.raises(bb.BigIntGPUError):
        bb.reciprocal_digits(np.array([1 << 28], dtype=np.uint32))  # not a 28-bit digit


def test_repeat_calls_reuse_buffers(bb, ref):
    """Large then small then large again through the same device buffers."""
    rng = np.random.default_rng(SEED + 402)
    for bits in (1 << 18, 1 << 8, 1 << 17, 1 << 18):
        check(bb, ref, rand_limbs(rng, bits // 64), 5, True, 0)
