"""The CPU oracle (oracle/bigint_oracle.c) pinned against the reference:
first against the committed golden vectors (made by running the reference),
then -- where oracle/_ref is built -- directly on fresh seeded inputs."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED, golden_digit_cases, golden_u64_cases, rand_digits, rand_limbs
from oracle.pyoracle import digits28_to_limbs, int_to_limbs, limbs_to_int


def test_port_matches_golden_u64(port, golden):
    n = 0
    for kind, a, b, c in golden_u64_cases(golden):
        got = port.ntt_mul(a, b) if b is not None else port.ntt_mul(a)
        assert np.array_equal(got, c), kind
        got = port.mul(a, b) if b is not None else port.mul(a)
        assert np.array_equal(got, c), kind
        n += 1
    assert n >= 20


def test_port_matches_golden_mul_digits(port, golden):
    n = 0
    for a, b, prec, pos, c in golden_digit_cases(golden):
        res, p = port.mul_digits(a, b, prec, 7)
        assert np.array_equal(res, c) and p == pos, (a.size, None if b is None else b.size, prec)
        n += 1
    assert n >= 40


def test_port_matches_golden_tree(port, golden):
    for k in range(2):
        leaves = golden[f"tree_{k:03d}_leaves"]
        want = digits28_to_limbs(golden[f"tree_{k:03d}_digits"])
        assert np.array_equal(port.product_tree(leaves), want)


def test_brute_equals_python_int(port):
    rng = np.random.default_rng(SEED + 1)
    for na, nb in [(1, 1), (2, 7), (31, 33), (128, 128)]:
        a, b = rand_limbs(rng, na), rand_limbs(rng, nb)
        want = int_to_limbs(limbs_to_int(a) * limbs_to_int(b))
        assert np.array_equal(port.brute_mul(a, b), want)


def test_mod_m61_residue_identity(port):
    rng = np.random.default_rng(SEED + 2)
    M = (1 << 61) - 1
    for n in [1, 5, 1000]:
        a = rand_limbs(rng, n)
        assert port.mod_m61(a) == limbs_to_int(a) % M


def test_zero_operand_gives_empty(port):
    z = np.zeros(3, dtype=np.uint64)
    assert port.ntt_mul(z, np.array([5], dtype=np.uint64)).size == 0


def test_port_matches_reference_random(port, reference):
    rng = np.random.default_rng(SEED + 3)
    for na, nb in [(1, 2), (200, 300), (2000, 1500), (9000, 9000), (20000, 313)]:
        a, b = rand_limbs(rng, na), rand_limbs(rng, nb)
        assert np.array_equal(port.ntt_mul(a, b), reference.ntt_mul(a, b))
        assert np.array_equal(port.mul(a), reference.mul(a))


def test_port_matches_reference_digits(port, reference):
    rng = np.random.default_rng(SEED + 4)
    for na, nb in [(7, 9), (5000, 3000)]:
        a, b = rand_digits(rng, na), rand_digits(rng, nb)
        for prec in (0, 3, 1000):
            assert np.array_equal(*(x[0] for x in (port.mul_digits(a, b, prec, 0),
                                                   reference.mul_digits(a, b, prec, 0))))


@pytest.mark.parametrize("n", [1, 64, 5000])
def test_port_all_ones_square(port, reference, n):
    ones = np.full(n, np.uint64(0xFFFFFFFFFFFFFFFF))
    assert np.array_equal(port.ntt_mul(ones), reference.ntt_mul(ones))
