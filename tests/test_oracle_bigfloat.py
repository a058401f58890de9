"""The step model of the device reciprocal, divmod and BigFloat print
(oracle/bigfloat_model.py) against the reference's own BigFloat::reciprocal
(src/bigint.cpp:1044-1071), BigInt::divmod (:625-673) and BigFloat::print
(:972-1041), on CPU: the way the device truncates products
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


def test_bigfloat_print_model_matches_reference(ref):
    """The print steps (fraction times 5^d, shift, rounding half up, carry)
    against BigFloat::print; inputs where the reference's rounding is
    undefined (the scaled fraction in [2^-28, 1/2)) are skipped."""
    import math

    from oracle import bigfloat_model as m
    from oracle.pyoracle import digits28_to_limbs

    if not ref.has_bigfloat_print:
        pytest.skip("reference oracle library without ref_bigfloat_print")
    rng = np.random.default_rng(SEED + 703)
    checked = 0
    for trial in range(300):
        bits = int(rng.integers(1, 400))
        x = int.from_bytes(rng.integers(0, 2**64, (bits + 63) // 64, dtype=np.uint64).tobytes(), "little")
        x = (x & ((1 << bits) - 1)) | (1 << (bits - 1))
        if trial % 9 == 0:  # a fraction just below an integer: rounds up and carries
            x = (x << 60) | ((1 << 60) - 1)
        offset = int(rng.integers(-500, 100))
        dec = [0, 0, 1, 3, 12, 40][trial % 6]
        xd = m._digits(x, (x.bit_length() + 27) // 28)
        # the BigFloat(X, offset) fields, computed exactly
        q = -(offset // 28) if offset < 0 else 0
        v = x << (offset + 28 * q)
        dd = m._digits(v, (v.bit_length() + 27) // 28)
        t = 0
        while dd[t] == 0:
            t += 1
        dd, pp = dd[t:], q - t
        dd_dec = dec or math.floor(float((min(pp, len(dd)) if pp > 0 else 0) * 28) * math.log10(2))
        if pp > 0 and dd_dec:
            frac = m._int(dd[: min(pp, len(dd))])
            scaled = frac * 10 ** dd_dec
            if frac and (scaled << 28) >= (1 << (28 * pp)) and 2 * scaled < (1 << (28 * pp)):
                continue  # the reference is undefined here
        (din, ppin), want = ref.bigfloat_print(digits28_to_limbs(np.array(xd, dtype=np.uint32)), offset,
                                               bool(trial & 1), dec)
        assert [int(y) for y in din] == dd and ppin == pp
        assert m.bigfloat_print(dd, pp, bool(trial & 1), dec) == want, (trial, bits, offset, dec)
        checked += 1
    assert checked > 200
