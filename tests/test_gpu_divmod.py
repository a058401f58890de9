"""BigInt::divmod on the GPU (bgpu_divmod_digits) against the reference's own
divmod (src/bigint.cpp:625-673): quotient and remainder Digits and signs
identical, for every rounding mode, every sign combination, with and without
the check, from single digits to NTT-sized operands.

Where the reference's conversion of its estimate is undefined (|A / B| in
[2^-28, 1]) the device result is checked against exact integer division with
the mode's rounding; at sizes where the reference is slow, against the
identity A = Q * B + R and the remainder's bound, by residues mod 2^61 - 1."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED

pytestmark = pytest.mark.gpu
MODES = (0, 1, 2, 3)  # Truncate, Floor, Ceil, RoundHalfUp
M61 = (1 << 61) - 1


@pytest.fixture(scope="module")
def ref():
    from oracle.pyoracle import Reference, have_reference

    if not have_reference():
        pytest.skip("reference oracle library not built")
    r = Reference()
    if not r.has_divmod:
        pytest.skip("reference oracle library without ref_divmod")
    return r


def rand_int_digits(rng, n: int) -> np.ndarray:
    d = rng.integers(0, 1 << 28, n, dtype=np.uint32)
    d[-1] = 1 + d[-1] % ((1 << 28) - 1)
    return d


def to_int(d) -> int:
    return sum(int(x) << (28 * i) for i, x in enumerate(d))


def from_int(v: int) -> np.ndarray:
    out = []
    while True:
        out.append(v & ((1 << 28) - 1))
        v >>= 28
        if not v:
            return np.array(out, dtype=np.uint32)


def ref_divmod(ref, a, a_neg, b, b_neg, mode, check=True):
    from oracle.pyoracle import digits28_to_limbs

    return ref.divmod(digits28_to_limbs(a), a_neg, digits28_to_limbs(b), b_neg, mode, check)


def check_vs_ref(bb, ref, a, a_neg, b, b_neg, mode, check=True):
    (q, qn), (r, rn) = bb.divmod_digits(a, b, a_neg, b_neg, mode, check)
    (wq, wqn), (wr, wrn) = ref_divmod(ref, a, a_neg, b, b_neg, mode, check)
    ctx = (a.size, b.size, a_neg, b_neg, mode, check)
    assert np.array_equal(q, wq) and qn == wqn, ctx
    assert np.array_equal(r, wr) and rn == wrn, ctx


def exact(av: int, bv: int, mode: int):
    """Python integer division with the reference's rounding modes."""
    fl = av // bv
    if mode == 1:
        q = fl
    elif mode == 2:
        q = -((-av) // bv)
    elif mode == 3:  # nearest, halves away from zero
        q2, r2 = divmod(2 * abs(av) + abs(bv), 2 * abs(bv))
        q = q2 if (av < 0) == (bv < 0) else -q2
    else:
        q = abs(av) // abs(bv)
        q = q if (av < 0) == (bv < 0) else -q
    return q, av - q * bv


def test_small_all_modes_and_signs(bb, ref):
    rng = np.random.default_rng(SEED + 800)
    for trial in range(120):
        nb = int(rng.integers(1, 6))
        na = nb + int(rng.integers(2, 8))
        a, b = rand_int_digits(rng, na), rand_int_digits(rng, nb)
        if trial % 7 == 0:
            a[: na // 2] = 0  # bottom zero digits (BigFloat(a) drops them)
        if trial % 11 == 0:
            b[: nb - 1] = 0
        for mode in MODES:
            check_vs_ref(bb, ref, a, bool(trial & 1), b, bool(trial & 2), mode)


def test_without_the_check(bb, ref):
    rng = np.random.default_rng(SEED + 801)
    for trial in range(30):
        nb = int(rng.integers(1, 40))
        a, b = rand_int_digits(rng, nb + int(rng.integers(2, 60))), rand_int_digits(rng, nb)
        check_vs_ref(bb, ref, a, bool(trial & 1), b, bool(trial & 2), trial % 4, check=False)


def test_exact_quotients_and_half_remainders(bb, ref):
    """R = 0 (the check is skipped) and |2R| = |B| (RoundHalfUp's tie)."""
    rng = np.random.default_rng(SEED + 802)
    for trial in range(24):
        b = rand_int_digits(rng, int(rng.integers(1, 30)))
        c = rand_int_digits(rng, int(rng.integers(2, 30)))
        bv, cv = to_int(b), to_int(c)
        a_exact = from_int(bv * cv)
        for mode in MODES:
            check_vs_ref(bb, ref, a_exact, bool(trial & 1), b, bool(trial & 2), mode)
        if bv % 2 == 0:
            a_half = from_int(bv * cv + bv // 2)
            for mode in MODES:
                check_vs_ref(bb, ref, a_half, bool(trial & 1), b, bool(trial & 2), mode)


def test_ntt_sized_operands(bb, ref):
    """Products inside the division on the NTT (tens of thousands of digits)."""
    rng = np.random.default_rng(SEED + 803)
    for na, nb in [(60000, 30000), (45000, 4000), (80000, 10), (40000, 20001)]:
        a, b = rand_int_digits(rng, na), rand_int_digits(rng, nb)
        for mode in (0, 1):
            check_vs_ref(bb, ref, a, mode == 1, b, False, mode)


def test_power_of_ten_split_like_print(bb, ref):
    """print_dec's call: a value divided by 10^k, k about half its decimal length."""
    rng = np.random.default_rng(SEED + 804)
    for nd in (500, 5000, 37450):
        a = rand_int_digits(rng, nd)
        k = int(np.ceil(nd * 28 * np.log10(2))) // 2
        p = from_int(10 ** k)
        check_vs_ref(bb, ref, a, False, p, False, 0)


def test_quotients_below_one_and_equal_operands(bb):
    """|A / B| <= 1: exact division with the mode's rounding (the reference's
    conversion is undefined there)."""
    rng = np.random.default_rng(SEED + 805)
    for trial in range(60):
        n = int(rng.integers(1, 8))
        a, b = rand_int_digits(rng, n), rand_int_digits(rng, n)
        if to_int(a) > to_int(b):
            a, b = b, a
        if trial % 5 == 0:
            a = b.copy()
        an, bn = bool(trial & 1), bool(trial & 2)
        for mode in MODES:
            (q, qn), (r, rn) = bb.divmod_digits(a, b, an, bn, mode)
            av, bv = (-1 if an else 1) * to_int(a), (-1 if bn else 1) * to_int(b)
            wq, wr = exact(av, bv, mode)
            assert (-1 if qn else 1) * to_int(q) == wq and (-1 if rn else 1) * to_int(r) == wr, (trial, mode)
            assert not (qn and to_int(q) == 0) and not (rn and to_int(r) == 0)


def test_zero_dividend_and_zero_divisor(bb):
    (q, qn), (r, rn) = bb.divmod_digits(np.array([0], np.uint32), np.array([7], np.uint32), True, True, 2)
    assert q.tolist() == [0] and r.tolist() == [0] and not qn and not rn
    with pytest.raises(bb.BigIntGPUError):
        bb.divmod_digits(np.array([5], np.uint32), np.array([0], np.uint32))


def mod_m61(d) -> int:
    v = 0
    for x in reversed(np.asarray(d, dtype=np.uint64).tolist()):
        v = ((v << 28) + x) % M61
    return v


def test_large_identity(bb):
    """2^22-bit / 2^21-bit: A = Q * B + R (mod 2^61 - 1) and 0 <= R < B."""
    rng = np.random.default_rng(SEED + 806)
    a, b = rand_int_digits(rng, (1 << 22) // 28), rand_int_digits(rng, (1 << 21) // 28)
    (q, qn), (r, rn) = bb.divmod_digits(a, b, False, False, 1)
    assert not qn and not rn
    assert (mod_m61(q) * mod_m61(b) + mod_m61(r)) % M61 == mod_m61(a)
    assert r.size < b.size or (r.size == b.size and r[::-1].tolist() < b[::-1].tolist())


def test_small_output_buffers_report_the_lengths_needed(bb):
    """BGPU_ERR_OUT_CAPACITY with *q_len and *r_len set, then a call with
    those capacities succeeds."""
    import ctypes as C

    rng = np.random.default_rng(SEED + 807)
    a, b = rand_int_digits(rng, 300), rand_int_digits(rng, 120)
    (wq, _), (wr, _) = bb.divmod_digits(a, b)
    u32p = C.POINTER(C.c_uint32)
    q, r = np.zeros(4, np.uint32), np.zeros(4, np.uint32)
    nq, nr, qn, rn = C.c_size_t(0), C.c_size_t(0), C.c_int(0), C.c_int(0)
    rc = bb.lib.bgpu_divmod_digits(a.ctypes.data_as(u32p), a.size, 0, b.ctypes.data_as(u32p), b.size, 0, 0, 1,
                                   q.ctypes.data_as(u32p), q.size, C.byref(nq), C.byref(qn),
                                   r.ctypes.data_as(u32p), r.size, C.byref(nr), C.byref(rn))
    assert rc == -5 and nq.value == wq.size and nr.value == wr.size
    q, r = np.zeros(nq.value, np.uint32), np.zeros(nr.value, np.uint32)
    rc = bb.lib.bgpu_divmod_digits(a.ctypes.data_as(u32p), a.size, 0, b.ctypes.data_as(u32p), b.size, 0, 0, 1,
                                   q.ctypes.data_as(u32p), q.size, C.byref(nq), C.byref(qn),
                                   r.ctypes.data_as(u32p), r.size, C.byref(nr), C.byref(rn))
    assert rc == 0 and np.array_equal(q, wq) and np.array_equal(r, wr)
    text = bb.bigfloat_to_decimal(a, 100, True, 30)
    buf, n = C.create_string_buffer(8), C.c_size_t(0)
    rc = bb.lib.bgpu_bigfloat_to_decimal(a.ctypes.data_as(u32p), a.size, 100, 1, 30, buf, 8, C.byref(n))
    assert rc == -5 and n.value == len(text)


def test_invalid_digits_are_rejected(bb):
    with pytest.raises(bb.BigIntGPUError):
        bb.divmod_digits(np.array([1 << 28], np.uint32), np.array([3], np.uint32))
    with pytest.raises(bb.BigIntGPUError):
        bb.divmod_digits(np.array([5, 0], np.uint32), np.array([3], np.uint32))  # a leading zero digit
    with pytest.raises(bb.BigIntGPUError):
        bb.bigfloat_to_decimal(np.array([3, 0], np.uint32), 1)
