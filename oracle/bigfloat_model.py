"""Step model of the device-resident reciprocal (test infrastructure only).

A pure-Python restatement, on Python integers, of the steps the engine runs
on the GPU for ``bgpu_reciprocal_digits`` (bigint_b200/csrc/engine.cu), which
replay the reference's BigFloat::reciprocal (src/bigint.cpp:1044-1071):

* ``mul_trunc`` -- BigFloat::mul with the truncation of mul_digits
  (include/bigint/mul.h:227-243, 301-312), computed the device's way: the
  truncated operands keep any zero digits at their bottom, and the first
  nonzero digit at or above the cut (``hi - prec`` for the two possible
  product lengths) is the result's bottom;
* ``add_or_sub`` -- BigFloat::add_or_sub (src/bigint.cpp:849-936) as the exact
  sum or difference in the reference's frame, leading and bottom zeros
  removed;
* ``shift``, ``to_double``, ``from_double`` -- src/bigint.cpp:681-812;
* ``divmod`` -- BigInt::divmod (src/bigint.cpp:625-673) as the engine replays
  it for ``bgpu_divmod_digits``: the estimate through ``reciprocal`` and
  ``mul_trunc``, its rounding to an integer (BigInt(const BigFloat&, mode),
  src/bigint.cpp:1072-1172), R = a - Q * b and the single adjustment;
* ``bigfloat_print`` -- BigFloat::print (src/bigint.cpp:972-1041) as the engine
  replays it for ``bgpu_bigfloat_to_decimal``: the fraction times 5^d, the
  shift by d - 28 pp, the rounding half up and the carry into the integer
  part.

tests/test_oracle_bigfloat.py pins this model against the reference's own
reciprocal, divmod and print; the GPU tests pin the device against the
reference.  Only the
tests import this module.
"""
from __future__ import annotations

import struct

MASK = (1 << 28) - 1


def _int(d):
    return sum(int(x) << (28 * i) for i, x in enumerate(d))


def _digits(v: int, n: int):
    return [(v >> (28 * i)) & MASK for i in range(n)]


def _ctrunc_div(a: int, b: int) -> int:  # C++ integer division (toward zero)
    q = abs(a) // b
    return q if a >= 0 else -q


class Val:
    """A BigFloat: digits (28-bit, little endian), point position, sign."""

    def __init__(self, d, pp: int, neg: bool):
        self.d, self.pp, self.neg = [int(x) for x in d], int(pp), bool(neg)

    def zero(self) -> bool:
        return len(self.d) == 1 and self.d[0] == 0

    def tz(self) -> int:
        t = 0
        while t < len(self.d) and self.d[t] == 0:
            t += 1
        return t


def plan_shift(pp: int, offset: int, low: int):
    """BigFloat::shift's choice (src/bigint.cpp:769-789): (pp, mode, s)."""
    pp -= _ctrunc_div(offset, 28)
    o = offset - _ctrunc_div(offset, 28) * 28
    if o == 0:
        return pp, 0, 0
    if o > 0:
        o = 28 - o
        pp -= 1
    else:
        o = -o
    ctz = (low & -low).bit_length() - 1 if low else 32
    if ctz >= o:
        return pp, 1, o
    return pp + 1, 2, 28 - o


def shift(v: Val, offset: int) -> Val:
    pp, mode, s = plan_shift(v.pp, offset, v.d[0])
    d, n = list(v.d), len(v.d)
    if mode == 1:
        d = [((d[i] >> s) | ((d[i + 1] << (28 - s)) if i + 1 < n else 0)) & MASK for i in range(n)]
    elif mode == 2:
        d = [(((d[i] << s) if i < n else 0) | ((d[i - 1] >> (28 - s)) if i > 0 else 0)) & MASK
             for i in range(n + 1)]
    while len(d) > 1 and d[-1] == 0:
        d.pop()
    neg = v.neg
    if len(d) == 1 and d[0] == 0:
        pp, neg = 0, False
    return Val(d, pp, neg)


def mul_trunc(a: Val, b: Val, prec: int) -> Val:
    if a.zero() or b.zero():
        return Val([0], 0, False)
    oa = len(a.d) - prec if len(a.d) > prec else 0
    ob = len(b.d) - prec if len(b.d) > prec else 0
    la, lb = len(a.d) - oa, len(b.d) - ob
    res = _digits(_int(a.d[oa:]) * _int(b.d[ob:]), la + lb + 1)
    hi = max(i for i, x in enumerate(res) if x) + 1
    assert hi in (la + lb - 1, la + lb)
    cut = hi - prec if hi > prec else 0
    first = min(i for i in range(cut, hi) if res[i])
    return Val(res[first:hi], a.pp + b.pp - (oa + ob + first), a.neg != b.neg)


def add_or_sub(a: Val, b: Val, is_sub: bool) -> Val:
    if a.zero():
        return Val(b.d, b.pp, (not b.neg) if (is_sub and not b.zero()) else b.neg)
    if b.zero():
        return a
    ppr = max(a.pp - a.tz(), b.pp - b.tz())
    length = max(len(a.d) - a.pp, len(b.d) - b.pp) + ppr
    A = _int(a.d) << (28 * (ppr - a.pp)) if ppr >= a.pp else _int(a.d) >> (28 * (a.pp - ppr))
    B = _int(b.d) << (28 * (ppr - b.pp)) if ppr >= b.pp else _int(b.d) >> (28 * (b.pp - ppr))
    neg = a.neg
    if a.neg != (b.neg != is_sub):
        if A == B:
            return Val([0], 0, False)
        if B > A:
            A, B, neg = B, A, not neg
        r = A - B
    else:
        r = A + B
    res = _digits(r, length + 1)
    hi = max(i for i, x in enumerate(res) if x) + 1
    lo = min(i for i, x in enumerate(res) if x)
    return Val(res[lo:hi], ppr - lo, neg)


def to_double(b: Val) -> float:
    n, top = len(b.d), b.d[-1]
    hbw = top.bit_length()
    e = 28 * (n - 1 - b.pp) + hbw - 1
    off = 52 - (hbw - 1)
    mant = (top & ((1 << (hbw - 1)) - 1)) << off
    i = n - 1
    while off > 0 and i > 0:
        off -= 28
        i -= 1
        mant |= b.d[i] >> -off if off < 0 else b.d[i] << off
    return struct.unpack("<d", struct.pack("<Q", (int(b.neg) << 63) | ((e + 1023) << 52) | mant))[0]


def from_double(v: float) -> Val:
    raw = struct.unpack("<Q", struct.pack("<d", v))[0]
    neg, eb, base = bool(raw >> 63), (raw >> 52) & 2047, raw & ((1 << 52) - 1)
    off = -52 - 1023
    if eb == 0:
        off += 1
    else:
        base |= 1 << 52
        off += eb
    d = []
    while base:
        d.append(base & MASK)
        base >>= 28
    return shift(Val(d, 0, neg), off)


def reciprocal(digits, pp: int, neg: bool, precision: int) -> Val:
    d = [int(x) for x in digits]
    if precision == 0:
        precision = len(d)
    expo = 28 * (len(d) - 1 - pp) + d[-1].bit_length()
    b = shift(Val(d, pp, neg), -expo)
    t = b.tz()
    b = Val(b.d[t:], b.pp - t, b.neg)
    x = from_double(1 / to_double(b))
    one = Val([1], 0, False)
    cur = 52 // 28
    while cur < precision:
        cur *= 2
        t1 = mul_trunc(b, x, cur + 1)
        t2 = add_or_sub(one, t1, True)
        t3 = mul_trunc(x, t2, cur + 1)
        x = add_or_sub(x, t3, False)
    return shift(x, -expo)


def _bigfloat_of_int(d, neg: bool) -> Val:
    """BigFloat(BigInt) (include/bigint/bigint.h:382-388): tail zeros removed."""
    d = [int(x) for x in d]
    if len(d) == 1 and d[0] == 0:
        return Val([0], 0, False)
    t = 0
    while d[t] == 0:
        t += 1
    return Val(d[t:], -t, neg)


def _signed(v: Val) -> int:
    """The integer value of a Val whose point position is <= 0."""
    if v.zero():
        return 0
    return (-1 if v.neg else 1) * (_int(v.d) << (28 * -v.pp))


def divmod(a, a_neg: bool, b, b_neg: bool, mode: int, check: bool = True):
    """(Q, R) as Python integers.  mode: 0 Truncate, 1 Floor, 2 Ceil,
    3 RoundHalfUp (others act as Truncate).  Where the reference's rounding
    of the estimate leaves no digits (2^-28 <= |estimate| < 1, nothing added),
    Q starts from zero, as on the device."""
    A, B = _bigfloat_of_int(a, a_neg), _bigfloat_of_int(b, b_neg)
    if B.zero():
        raise ZeroDivisionError("division by zero")
    if A.zero():
        return 0, 0
    prec = len(a) + 16
    p = mul_trunc(A, reciprocal(B.d, B.pp, B.neg, prec), prec)
    if p.zero() or p.pp > len(p.d):
        q = 0
    elif p.pp <= 0:
        q = _signed(p)
    else:
        k = p.pp  # digits below the point; p.d[0] != 0
        inc = {1: p.neg, 2: not p.neg, 3: bool(p.d[k - 1] >> 27)}.get(mode, False)
        mag = (_int(p.d[k:]) if k < len(p.d) else 0) + int(inc)
        q = -mag if p.neg else mag
    av, bv = _signed(A), _signed(B)
    r = av - q * bv
    if check and r != 0:
        rn, bn, an = r < 0, bv < 0, av < 0
        if mode == 3:
            c = (abs(2 * r) > abs(bv)) - (abs(2 * r) < abs(bv))
            adjust = c > 0 or (c == 0 and rn == an)
        else:
            over = abs(r) >= abs(bv)
            adjust = {1: rn != bn or over, 2: rn == bn or over}.get(mode, rn != an or over)
        if adjust:
            if rn != bn:
                r, q = r + bv, q - 1
            else:
                r, q = r - bv, q + 1
    return q, r


def _round_half_up_to_int(p: Val) -> int:
    """BigInt(const BigFloat&, RoundHalfUp) of a Val whose bottom digit is
    nonzero, as the device computes it; zero where the reference's rounding
    leaves no digit."""
    if p.zero() or p.pp > len(p.d):
        return 0
    if p.pp <= 0:
        return _signed(p)
    k = p.pp
    mag = (_int(p.d[k:]) if k < len(p.d) else 0) + (p.d[k - 1] >> 27)
    return -mag if p.neg else mag


def bigfloat_print(digits, pp: int, neg: bool, dec_digits: int = 0) -> str:
    """The text of BigFloat::print(out, dec_digits) for a BigFloat's fields."""
    import math
    import sys

    d = [int(x) for x in digits]
    n = len(d)
    int_part = (_int(d[max(pp, 0):]) << (28 * max(-pp, 0))) if pp < n else 0
    fsize = min(pp, n) if pp > 0 else 0
    if dec_digits == 0:
        dec_digits = math.floor(float(fsize * 28) * math.log10(2))
    frac = _int(d[:fsize])
    f = 0
    if dec_digits and frac:
        x = frac * 5 ** dec_digits
        xd = _digits(x, (x.bit_length() + 27) // 28)
        t = 0
        while xd[t] == 0:
            t += 1
        s = shift(Val(xd[t:], -t, False), dec_digits - 28 * pp)
        t = s.tz()
        f = _round_half_up_to_int(Val(s.d[t:], s.pp - t, False))
        if f == 10 ** dec_digits:
            f, int_part = 0, int_part + 1
    old = sys.get_int_max_str_digits()
    sys.set_int_max_str_digits(0)
    try:
        text = ("-" if neg else "") + str(int_part) + "."
        if dec_digits:
            text += str(f).rjust(dec_digits, "0")
    finally:
        sys.set_int_max_str_digits(old)
    return text
