"""The reference's own, unmodified BigInt / BigFloat code running its products
on this engine: the reference built without its CPU NTT and FFT translation
units and with bigint_b200/hooks/reference_hook.cpp in their place (the
link-time drop-in a maintainer of the reference would use).  Every result is compared with the pure
reference library on the same inputs."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED, rand_digits, rand_limbs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("na,nb", [(100, 100), (1000, 3000), (40000, 40000), (100000, 100000),
                                   (250000, 3000), (1, 200000)])
def test_dispatch_products(bb, reference, reference_gpu, na, nb):
    """_mul routes these to brute (inline, CPU), fft::mul and ntt::mul (hooked)."""
    rng = np.random.default_rng(SEED + 90 + na + nb)
    a, b = rand_limbs(rng, na), rand_limbs(rng, nb)
    assert np.array_equal(reference_gpu.mul(a, b), reference.mul(a, b))
    assert np.array_equal(reference_gpu.mul(a), reference.mul(a))  # squaring by pointer identity
    ones = np.full(na, np.uint64(0xFFFFFFFFFFFFFFFF))
    assert np.array_equal(reference_gpu.ntt_mul(ones), reference.ntt_mul(ones))


def test_mul_digits_precision(bb, reference, reference_gpu):
    rng = np.random.default_rng(SEED + 91)
    for nd, prec in [(50000, 0), (50000, 20000), (300000, 1000), (7, 0)]:
        a, b = rand_digits(rng, nd), rand_digits(rng, nd // 2 + 3)
        assert np.array_equal(*(r.mul_digits(a, b, prec, 5)[0] for r in (reference_gpu, reference)))
        ra, pa = reference_gpu.mul_digits(a, b, prec, 5)
        rb, pb = reference.mul_digits(a, b, prec, 5)
        assert np.array_equal(ra, rb) and pa == pb


def test_bigint_product_tree(bb, reference, reference_gpu):
    rng = np.random.default_rng(SEED + 92)
    leaves = rng.integers(1 << 32, 2**64, 1 << 14, dtype=np.uint64, endpoint=False)
    assert np.array_equal(reference_gpu.product_tree_digits(leaves), reference.product_tree_digits(leaves))


def test_fast_pow(bb, reference, reference_gpu):
    if not reference.has_fast_pow:
        pytest.skip("reference shim without fast_pow")
    assert np.array_equal(reference_gpu.fast_pow_digits(1234567, 100003),
                          reference.fast_pow_digits(1234567, 100003))


@pytest.mark.parametrize("nleaves,prec", [(1024, 500), (1024, 50000), (16384, 200000)])
def test_bigfloat_reciprocal(bb, reference, reference_gpu, nleaves, prec):
    """BigFloat::reciprocal's Newton iteration (src/bigint.cpp:1044-1071):
    its BigFloat::mul products go through mul_digits -> _mul -> the hook."""
    if not reference.has_reciprocal:
        pytest.skip("reference shim without reciprocal")
    rng = np.random.default_rng(SEED + 93 + nleaves)
    leaves = rng.integers(1 << 32, 2**64, nleaves, dtype=np.uint64, endpoint=False)
    dg, pg = reference_gpu.reciprocal_digits(leaves, prec)
    dr, pr = reference.reciprocal_digits(leaves, prec)
    assert pg == pr and np.array_equal(dg, dr)


@pytest.mark.parametrize("nlimbs", [1000, 16384])
def test_decimal_print(bb, reference, reference_gpu, nlimbs):
    """BigInt::print (src/bigint.cpp:175-247): print_dec's divmod and
    get_pow_of_ten products go through the hook; the decimal text must not
    change."""
    if not reference.has_to_dec:
        pytest.skip("reference shim without ref_to_dec_string")
    rng = np.random.default_rng(SEED + 94 + nlimbs)
    limbs = rng.integers(0, 2**64, nlimbs, dtype=np.uint64)
    limbs[-1] |= np.uint64(1 << 63)
    text = reference_gpu.to_dec_string(limbs)
    assert text == reference.to_dec_string(limbs)
    if nlimbs == 1000:  # small enough for Python's own conversion
        import sys

        old = sys.get_int_max_str_digits()
        sys.set_int_max_str_digits(0)
        try:
            assert text == str(int.from_bytes(limbs.tobytes(), "little"))
        finally:
            sys.set_int_max_str_digits(old)
