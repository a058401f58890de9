"""Decimal text to BigInt on the GPU (bgpu_from_decimal) against the
reference's BigInt(const std::string&) (src/bigint.cpp:25-124): Digits and
sign identical, including the reference's handling of signs, stray
characters, leading zeros and zero."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    from oracle.pyoracle import Reference, have_reference

    if not have_reference():
        pytest.skip("reference oracle library not built")
    r = Reference()
    if not r.has_from_dec:
        pytest.skip("reference oracle library without ref_from_dec_string")
    return r


def check(bb, ref, text: bytes):
    got, neg = bb.from_decimal(text)
    want, wneg = ref.from_dec_string(text)
    assert neg == wneg and np.array_equal(got, want), (text[:40], len(text), got.size, want.size)


def test_edge_strings(bb, ref):
    for t in [b"0", b"-0", b"", b"-", b"--5", b"+7", b"  -12a3", b"1", b"9" * 19, b"1" + b"0" * 19,
              b"0000123456789012345678901234567890", b"12,345,678,901,234,567,890,123", b"-" + b"9" * 40,
              b"x1y2z3"]:
        check(bb, ref, t)


def test_sizes_across_leaves_and_levels(bb, ref):
    """Lengths around the 19-digit leaves, the 32-limb first segments and the
    level boundaries (19 * 2^j digits)."""
    rng = np.random.default_rng(SEED + 600)
    lengths = {1, 18, 19, 20, 37, 38, 39, 607, 608, 609, 1215, 1216, 1217}
    for j in range(5, 15):
        lengths |= {19 * (1 << j) - 1, 19 * (1 << j), 19 * (1 << j) + 1}
    for n in sorted(lengths):
        d = rng.integers(0, 10, n, dtype=np.uint8)
        d[0] = 1 + d[0] % 9
        check(bb, ref, (d + ord("0")).tobytes())


def test_all_nines_and_powers_of_ten(bb, ref):
    for n in (19 * 32, 19 * 1024, 100000):
        check(bb, ref, b"9" * n)
        check(bb, ref, b"1" + b"0" * n)


def test_matches_python_int(bb):
    import sys

    rng = np.random.default_rng(SEED + 601)
    d = rng.integers(0, 10, 5000, dtype=np.uint8)
    d[0] = 7
    text = (d + ord("0")).tobytes()
    old = sys.get_int_max_str_digits()
    sys.set_int_max_str_digits(0)
    try:
        v = int(text)
    finally:
        sys.set_int_max_str_digits(old)
    got, neg = bb.from_decimal(b"-" + text)
    assert neg
    assert sum(int(x) << (28 * i) for i, x in enumerate(got)) == v


def test_large(bb, ref):
    """1.26 M digits (a 2^22-bit value)."""
    rng = np.random.default_rng(SEED + 602)
    d = rng.integers(0, 10, 1262612, dtype=np.uint8)
    d[0] = 3
    check(bb, ref, (d + ord("0")).tobytes())
