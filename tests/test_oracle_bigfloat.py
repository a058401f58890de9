"""The step model of the device reciprocal and divmod (oracle/bigfloat_model.py)
against the reference's own BigFloat::reciprocal (src/bigint.cpp:1044-1071)
and BigInt::divmod (:625-673), on CPU: the way the device truncates products
(operands keep their bottom zeros, the cut lands on the first nonzero digit at
or above it) gives the reference's digits, point position and sign, and the
device's rounding of the quotient estimate and its adjustment give the
reference's quotient and remainder."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED


@pytest.fixture(scope="module")
def ref():
    from oracle.pyoracle import Reference, have_reference

    if not have_reference():
        pytest.skip("reference oracle library not built")
    r = Reference()
    if not r.has_bigfloat_reciprocal:
        pytest.skip("reference oracle library without ref_bigfloat_reciprocal")
    return r


def test_model_matches_reference(ref):
    from oracle import bigfloat_model as m

    rng = np.random.default_rng(SEED + 700)
    for trial in range(150):
        n = int(rng.integers(1, 6))
        limbs = rng.integers(1, 2**64, n, dtype=np.uint64)
        if trial % 5 == 0:
            limbs[:] = np.uint64(2**64 - 1)
        if trial % 6 == 0:
            limbs[:-1] = 0
            limbs[-1] = np.uint64(1 << int(rng.integers(0, 64)))
        offset, neg, prec = int(rng.integers(-300, 300)), bool(trial & 1), int(rng.integers(0, 60))
        (din, ppin, nin), (want, wpp, wneg) = ref.bigfloat_reciprocal(limbs, offset, neg, prec)
        got = m.reciprocal(din, ppin, nin, prec)
        assert got.d == [int(x) for x in want] and got.pp == wpp and got.neg == wneg, (trial, offset, prec)


def test_mul_trunc_matches_reference_mul_digits(ref):
    """The device-style truncation against the reference's mul_digits with
    output_precision, on operands whose cut falls on zero digits."""
    from oracle import bigfloat_model as m

    rng = np.random.default_rng(SEED + 701)
    for trial in range(200):
        na, nb = int(rng.integers(1, 12)), int(rng.integers(1, 12))
        a = rng.integers(0, 1 << 28, na, dtype=np.uint32)
        b = rng.integers(0, 1 << 28, nb, dtype=np.uint32)
        a[-1] |= 1
        b[-1] |= 1
        a[rng.random(na) < 0.4] = 0  # zero digits around the cut
        b[rng.random(nb) < 0.4] = 0
        a[-1] |= 1
        b[-1] |= 1
        if not a.any() or not b.any():
            continue
        prec = int(rng.integers(1, 14))
        want, wpos = ref.mul_digits(a, b, prec, 0)
        got = m.mul_trunc(m.Val(a, 0, False), m.Val(b, 0, False), prec)
        assert got.d == [int(x) for x in want] and got.pp == wpos, (trial, na, nb, prec)


def test_divmod_model_matches_reference(ref):
    from oracle import bigfloat_model as m
    from oracle.pyoracle import digits28_to_limbs

    if not ref.has_divmod:
        pytest.skip("reference oracle library without ref_divmod")
    rng = np.random.default_rng(SEED + 702)
    to_int = lambda d, neg: (-1 if neg else 1) * sum(int(x) << (28 * i) for i, x in enumerate(d))
    for trial in range(100):
        nb = int(rng.integers(1, 6))
        na = nb + int(rng.integers(2, 8))  # |a / b| >= 2^28: the reference is defined
        a = rng.integers(0, 1 << 28, na, dtype=np.uint32)
        b = rng.integers(0, 1 << 28, nb, dtype=np.uint32)
        a[-1] |= 1
        b[-1] |= 1
        if trial % 7 == 0:
            a[: na // 2] = 0
        an, bn = bool(trial & 1), bool(trial & 2)
        for mode in range(4):
            for check in (True, False):
                (q, qn), (r, rn) = ref.divmod(digits28_to_limbs(a), an, digits28_to_limbs(b), bn, mode, check)
                got = m.divmod(a, an, b, bn, mode, check)
                assert got == (to_int(q, qn), to_int(r, rn)), (trial, mode, check)
