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


# ---- BigInt to decimal text (bgpu_to_decimal) against BigInt::print ----------

def print_check(bb, ref, d, neg=False):
    from oracle.pyoracle import digits28_to_limbs

    got = bb.to_decimal(d, neg)
    limbs = digits28_to_limbs(d)
    want = ref.to_dec_string(limbs) if limbs.size else "0"
    if neg and want != "0":
        want = "-" + want
    assert got == want, (d.size, got[:30], want[:30], len(got), len(want))


def test_print_small_and_edges(bb, ref):
    for v in [0, 1, 9, 10, 10**19 - 1, 10**19, 10**19 + 1, 2**64 - 1, 2**64, 10**38, 10**57 - 1, 2**200]:
        d = np.array([(v >> (28 * i)) & ((1 << 28) - 1) for i in range(max(1, (v.bit_length() + 27) // 28))],
                     dtype=np.uint32)
        print_check(bb, ref, d)
        print_check(bb, ref, d, neg=True)


def test_print_sizes_across_levels(bb, ref):
    """Values whose decimal length crosses the printed leaves (608 digits)
    and each division level."""
    rng = np.random.default_rng(SEED + 610)
    for decimal_len in [100, 607, 608, 609, 1215, 1216, 1217, 2431, 2432, 2433, 4865, 9729, 20000, 77824, 77825, 155649,
                        400000]:
        nd = int(decimal_len / 0.30103 / 28) + 1
        d = rng.integers(0, 1 << 28, nd, dtype=np.uint32)
        d[-1] = 1 + d[-1] % ((1 << 27) - 1)
        print_check(bb, ref, d)


def test_print_powers_of_ten_and_ones(bb, ref):
    """10^k - 1, 10^k and all-ones Digits: quotient corrections at every level."""
    for k in (2432, 4864, 9728, 19456, 38912):
        text = "9" * k
        d, _ = bb.from_decimal(text)
        assert bb.to_decimal(d) == text
        d, _ = bb.from_decimal("1" + "0" * k)
        assert bb.to_decimal(d) == "1" + "0" * k
    print_check(bb, ref, np.full(30000, (1 << 28) - 1, dtype=np.uint32))


def test_print_round_trip_large(bb, ref):
    rng = np.random.default_rng(SEED + 611)
    dd = rng.integers(0, 10, 1262612, dtype=np.uint8)
    dd[0] = 5
    text = (dd + ord("0")).tobytes().decode()
    d, neg = bb.from_decimal(text)
    assert bb.to_decimal(d, neg) == text
    print_check(bb, ref, d)
