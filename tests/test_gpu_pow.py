"""fast_pow on the GPU (bgpu_pow_u64): the reference's squaring chain
(fast_pow<BigInt>, include/bigint/bigint_base.h:60-69) with every product on
the device, checked against Python's exact integer power and, where the
compiled reference is present, against the reference's own fast_pow."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED, rand_limbs
from oracle.pyoracle import digits28_to_limbs, int_to_limbs, limbs_to_int

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("base,e", [(1234567, 0), (1234567, 1), (1234567, 2), (1234567, 3),
                                    (1234567, 1000), (1234567, 65537), (3, 200003),
                                    (2**64 - 1, 5000), (2, 12345), (1, 99), (0, 0), (0, 7)])
def test_fast_pow_small_bases(bb, base, e):
    got = bb.fast_pow(base, e)
    assert limbs_to_int(got) == base**e, (base, e)
    want = int_to_limbs(base**e)
    assert got.size == want.size  # no leading zero limbs


def test_fast_pow_multi_limb_base(bb):
    rng = np.random.default_rng(SEED + 70)
    for n, e in [(3, 777), (40, 301), (1000, 17)]:
        a = rand_limbs(rng, n)
        assert limbs_to_int(bb.fast_pow(a, e)) == limbs_to_int(a) ** e, (n, e)


def test_fast_pow_matches_reference(bb, reference):
    if not reference.has_fast_pow:
        pytest.skip("compiled reference has no fast_pow entry point")
    want = digits28_to_limbs(reference.fast_pow_digits(1234567, 300007))
    assert np.array_equal(bb.fast_pow(1234567, 300007), want)


def test_fast_pow_benchmark_size_residue(bb, port):
    """1234567^7654321 (the reference's benchmark, examples/benchmark.cpp:22),
    about 155 Mbit: residue mod 2^61-1 by modular exponentiation."""
    m = (1 << 61) - 1
    got = bb.fast_pow(1234567, 7654321)
    assert port.mod_m61(got) == pow(1234567, 7654321, m)
    assert abs(got.size * 64 - 7654321 * np.log2(1234567)) < 128
