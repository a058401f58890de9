"""ctypes bindings for the CPU oracle (test infrastructure only).

``Port`` wraps ``oracle/liboracle.so`` (the C restatement); ``Reference``
wraps ``oracle/_ref/libbigint_ref.so`` (the unmodified reference compiled by
``oracle/build.py``).  Only the tests, ``__graft_entry__.smoke()`` and the
bench's CPU legs import this module; it is the checker, never the product.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libbigint_ref.so")
# The same reference sources with ntt::mul / fft::mul / init_thread_pool taken
# from bigint_b200/hooks/reference_hook.cpp (products on the GPU engine).
REF_GPU_SO = os.path.join(HERE, "_ref", "libbigint_ref_gpu.so")

_u64p = C.POINTER(C.c_uint64)
_u32p = C.POINTER(C.c_uint32)
_szp = C.POINTER(C.c_size_t)


def _p64(a: np.ndarray):
    return a.ctypes.data_as(_u64p)


def _p32(a: np.ndarray):
    return a.ctypes.data_as(_u32p)


class OracleError(RuntimeError):
    pass


def _limbs(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint64))


def _digits(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint32))


class _Lib:
    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library not built: {path} (run python oracle/build.py)")
        self.path = path
        self.lib = C.CDLL(path)

    def _mul64(self, fn, a, b, *extra, same: bool = False) -> np.ndarray:
        a = _limbs(a)
        b = a if same else _limbs(b)
        cap = a.size + b.size + 2
        out = np.zeros(max(cap, 1), dtype=np.uint64)
        n = C.c_size_t(0)
        pa = _p64(a) if a.size else _p64(np.zeros(1, np.uint64))
        pb = pa if same else (_p64(b) if b.size else _p64(np.zeros(1, np.uint64)))
        rc = fn(pa, a.size, pb, b.size, *extra, _p64(out), cap, C.byref(n))
        if rc != 0:
            raise OracleError(f"{fn.__name__} returned {rc}")
        return out[: n.value].copy()


class Port(_Lib):
    """The plain-C restatement (oracle/bigint_oracle.c)."""

    def __init__(self, path: str = PORT_SO):
        super().__init__(path)
        L = self.lib
        for name in ("orc_ntt_mul", "orc_brute_mul", "orc_mul"):
            f = getattr(L, name)
            f.argtypes = [_u64p, C.c_size_t, _u64p, C.c_size_t, _u64p, C.c_size_t, _szp]
            f.restype = C.c_int
        L.orc_mul_digits.argtypes = [_u32p, C.c_size_t, _u32p, C.c_size_t, C.c_int, C.c_size_t,
                                     C.POINTER(C.c_int64), _u32p, C.c_size_t, _szp]
        L.orc_mul_digits.restype = C.c_int
        L.orc_mod_m61.argtypes = [_u64p, C.c_size_t]
        L.orc_mod_m61.restype = C.c_uint64
        L.orc_product_tree.argtypes = [_u64p, C.c_size_t, _u64p, C.c_size_t, _szp]
        L.orc_product_tree.restype = C.c_int

    def ntt_mul(self, a, b=None) -> np.ndarray:
        return self._mul64(self.lib.orc_ntt_mul, a, b, same=b is None)

    def brute_mul(self, a, b=None) -> np.ndarray:
        return self._mul64(self.lib.orc_brute_mul, a, b, same=b is None)

    def mul(self, a, b=None) -> np.ndarray:
        return self._mul64(self.lib.orc_mul, a, b, same=b is None)

    def mul_digits(self, a, b=None, output_precision: int = 0, point_pos: int | None = None):
        return _mul_digits(self.lib.orc_mul_digits, a, b, output_precision, point_pos)

    def mod_m61(self, x) -> int:
        x = _limbs(x)
        if x.size == 0:
            return 0
        return int(self.lib.orc_mod_m61(_p64(x), x.size))

    def product_tree(self, leaves) -> np.ndarray:
        leaves = _limbs(leaves)
        cap = leaves.size + 2
        out = np.zeros(cap, dtype=np.uint64)
        n = C.c_size_t(0)
        rc = self.lib.orc_product_tree(_p64(leaves), leaves.size, _p64(out), cap, C.byref(n))
        if rc != 0:
            raise OracleError(f"orc_product_tree returned {rc}")
        return out[: n.value].copy()


def _mul_digits(fn, a, b, output_precision, point_pos):
    a = _digits(a)
    same = b is None
    b = a if same else _digits(b)
    cap = a.size + b.size + 4
    out = np.zeros(cap, dtype=np.uint32)
    n = C.c_size_t(0)
    pp = C.c_int64(point_pos if point_pos is not None else 0)
    rc = fn(_p32(a), a.size, _p32(b), b.size, int(same), int(output_precision),
            C.byref(pp) if point_pos is not None else None, _p32(out), cap, C.byref(n))
    if rc != 0:
        raise OracleError(f"mul_digits returned {rc}")
    res = out[: n.value].copy()
    if point_pos is not None:
        return res, int(pp.value)
    return res


class Reference(_Lib):
    """The unmodified reference path (oracle/_ref/libbigint_ref.so)."""

    def __init__(self, path: str = REF_SO):
        super().__init__(path)
        L = self.lib
        for name in ("ref_ntt_mul", "ref_ssa_mul", "ref_brute_mul", "ref_mul"):
            f = getattr(L, name)
            f.argtypes = [_u64p, C.c_size_t, _u64p, C.c_size_t, _u64p, C.c_size_t, _szp]
            f.restype = C.c_int
        L.ref_fft_mul.argtypes = [_u64p, C.c_size_t, _u64p, C.c_size_t, C.c_int, _u64p,
                                  C.c_size_t, _szp]
        L.ref_fft_mul.restype = C.c_int
        L.ref_mul_digits.argtypes = [_u32p, C.c_size_t, _u32p, C.c_size_t, C.c_int, C.c_size_t,
                                     C.POINTER(C.c_int64), _u32p, C.c_size_t, _szp]
        L.ref_mul_digits.restype = C.c_int
        L.ref_product_tree.argtypes = [_u64p, C.c_size_t, _u32p, C.c_size_t, _szp]
        L.ref_product_tree.restype = C.c_int
        L.ref_init_thread_pool.argtypes = [C.c_uint32]
        L.ref_init_thread_pool.restype = None
        self.has_bigfloat_reciprocal = hasattr(L, "ref_bigfloat_reciprocal")
        if self.has_bigfloat_reciprocal:
            L.ref_bigfloat_reciprocal.argtypes = [_u64p, C.c_size_t, C.c_int64, C.c_int, C.c_size_t,
                                                  _u32p, C.c_size_t, _szp, C.POINTER(C.c_int64),
                                                  _u32p, C.c_size_t, _szp, C.POINTER(C.c_int64),
                                                  C.POINTER(C.c_int)]
            L.ref_bigfloat_reciprocal.restype = C.c_int
        self.has_to_dec = hasattr(L, "ref_to_dec_string")
        if self.has_to_dec:
            L.ref_to_dec_string.argtypes = [_u64p, C.c_size_t, C.c_char_p, C.c_size_t, _szp]
            L.ref_to_dec_string.restype = C.c_int
        self.has_divmod = hasattr(L, "ref_divmod")
        if self.has_divmod:
            L.ref_divmod.argtypes = [_u64p, C.c_size_t, C.c_int, _u64p, C.c_size_t, C.c_int, C.c_uint32,
                                     C.c_int, _u32p, C.c_size_t, _szp, C.POINTER(C.c_int), _u32p,
                                     C.c_size_t, _szp, C.POINTER(C.c_int)]
            L.ref_divmod.restype = C.c_int
        self.has_bigfloat_print = hasattr(L, "ref_bigfloat_print")
        if self.has_bigfloat_print:
            L.ref_bigfloat_print.argtypes = [_u64p, C.c_size_t, C.c_int64, C.c_int, C.c_size_t, _u32p,
                                             C.c_size_t, _szp, C.POINTER(C.c_int64), C.c_char_p,
                                             C.c_size_t, _szp]
            L.ref_bigfloat_print.restype = C.c_int
        self.has_from_dec = hasattr(L, "ref_from_dec_string")
        if self.has_from_dec:
            L.ref_from_dec_string.argtypes = [C.c_char_p, C.c_size_t, _u32p, C.c_size_t, _szp,
                                              C.POINTER(C.c_int)]
            L.ref_from_dec_string.restype = C.c_int
        self.has_reciprocal = hasattr(L, "ref_reciprocal")
        if self.has_reciprocal:
            L.ref_reciprocal.argtypes = [_u64p, C.c_size_t, C.c_size_t, _u32p, C.c_size_t, _szp,
                                         C.POINTER(C.c_int64)]
            L.ref_reciprocal.restype = C.c_int
        self.has_fast_pow = hasattr(L, "ref_fast_pow")
        if self.has_fast_pow:
            L.ref_fast_pow.argtypes = [C.c_uint64, C.c_uint32, _u32p, C.c_size_t, _szp]
            L.ref_fast_pow.restype = C.c_int

    def init_thread_pool(self, n: int) -> None:
        """First call wins (ntt_multithread.cpp:287-290); 0/1 disables threads."""
        self.lib.ref_init_thread_pool(int(n))

    def ntt_mul(self, a, b=None) -> np.ndarray:
        return self._mul64(self.lib.ref_ntt_mul, a, b, same=b is None)

    def ssa_mul(self, a, b=None) -> np.ndarray:
        return self._mul64(self.lib.ref_ssa_mul, a, b, same=b is None)

    def brute_mul(self, a, b=None) -> np.ndarray:
        return self._mul64(self.lib.ref_brute_mul, a, b, same=b is None)

    def mul(self, a, b=None) -> np.ndarray:
        return self._mul64(self.lib.ref_mul, a, b, same=b is None)

    def fft_mul(self, a, b=None, digit_bits: int = 0) -> np.ndarray:
        return self._mul64(self.lib.ref_fft_mul, a, b, int(digit_bits), same=b is None)

    def mul_digits(self, a, b=None, output_precision: int = 0, point_pos: int | None = None):
        return _mul_digits(self.lib.ref_mul_digits, a, b, output_precision, point_pos)

    def reciprocal_digits(self, leaves, precision: int):
        """BigFloat(prod(leaves)).reciprocal(precision): (digits, point_pos)."""
        leaves = _limbs(leaves)
        n = C.c_size_t(0)
        pp = C.c_int64(0)
        cap = 4 * int(precision) + 64  # Newton's last step may leave up to ~2x precision digits
        out = np.zeros(cap, dtype=np.uint32)
        rc = self.lib.ref_reciprocal(_p64(leaves), leaves.size, int(precision), _p32(out), cap, C.byref(n),
                                     C.byref(pp))
        if rc != 0:
            raise OracleError(f"ref_reciprocal returned {rc}")
        return out[: n.value].copy(), int(pp.value)

    def bigfloat_reciprocal(self, limbs, offset: int, neg: bool, precision: int):
        """(+-BigFloat(X, offset)).reciprocal(precision), X = the integer with
        little-endian u64 ``limbs`` (nonzero).

        Returns ((in_digits, in_point_pos, neg), (digits, point_pos, neg)): the
        input BigFloat's fields and the reciprocal's."""
        leaves = _limbs(limbs)
        in_cap = (leaves.size * 64) // 28 + 8
        cap = 4 * max(int(precision), in_cap) + 64
        din = np.zeros(in_cap, dtype=np.uint32)
        out = np.zeros(cap, dtype=np.uint32)
        nin, nout = C.c_size_t(0), C.c_size_t(0)
        ppin, pp, oneg = C.c_int64(0), C.c_int64(0), C.c_int(0)
        rc = self.lib.ref_bigfloat_reciprocal(_p64(leaves), leaves.size, int(offset), int(bool(neg)),
                                              int(precision), _p32(din), in_cap, C.byref(nin),
                                              C.byref(ppin), _p32(out), cap, C.byref(nout), C.byref(pp),
                                              C.byref(oneg))
        if rc != 0:
            raise OracleError(f"ref_bigfloat_reciprocal returned {rc}")
        return ((din[: nin.value].copy(), int(ppin.value), bool(neg)),
                (out[: nout.value].copy(), int(pp.value), bool(oneg.value)))

    def divmod(self, a_limbs, a_neg: bool, b_limbs, b_neg: bool, mode: int = 0, check: bool = True):
        """(+-A).divmod(+-B, mode, check) for A, B given by little-endian u64
        limbs: ((Q Digits, Q negative), (R Digits, R negative)).  |A / B| must
        stay out of [2^-28, 1] (the reference's conversion is undefined there)."""
        la, lb = _limbs(a_limbs), _limbs(b_limbs)
        qcap = max(la.size - lb.size + 2, 1) * 3 + 8
        rcap = max(la.size, lb.size) * 3 + 8
        q, r = np.zeros(qcap, dtype=np.uint32), np.zeros(rcap, dtype=np.uint32)
        nq, nr, qn, rn = C.c_size_t(0), C.c_size_t(0), C.c_int(0), C.c_int(0)
        rc = self.lib.ref_divmod(_p64(la), la.size, int(bool(a_neg)), _p64(lb), lb.size, int(bool(b_neg)),
                                 int(mode), int(bool(check)), _p32(q), qcap, C.byref(nq), C.byref(qn),
                                 _p32(r), rcap, C.byref(nr), C.byref(rn))
        if rc != 0:
            raise OracleError(f"ref_divmod returned {rc}")
        return ((q[: nq.value].copy(), bool(qn.value)), (r[: nr.value].copy(), bool(rn.value)))

    def bigfloat_print(self, limbs, offset: int, neg: bool, dec_digits: int = 0):
        """(+-BigFloat(X, offset)).print(out, dec_digits) for X with
        little-endian u64 ``limbs``: ((in_digits, in_point_pos), text)."""
        leaves = _limbs(limbs)
        in_cap = (leaves.size * 64) // 28 + 8
        cap = int(in_cap * 9 + abs(int(offset)) * 0.31 + int(dec_digits)) + 64
        din = np.zeros(in_cap, dtype=np.uint32)
        out = C.create_string_buffer(cap)
        nin, nout, ppin = C.c_size_t(0), C.c_size_t(0), C.c_int64(0)
        rc = self.lib.ref_bigfloat_print(_p64(leaves), leaves.size, int(offset), int(bool(neg)), int(dec_digits),
                                         _p32(din), in_cap, C.byref(nin), C.byref(ppin), out, cap, C.byref(nout))
        if rc != 0:
            raise OracleError(f"ref_bigfloat_print returned {rc}")
        return (din[: nin.value].copy(), int(ppin.value)), out.raw[: nout.value].decode()

    def to_dec_string(self, limbs) -> str:
        """Decimal text of the integer with little-endian u64 ``limbs``
        (BigInt::print)."""
        leaves = _limbs(limbs)
        cap = int(leaves.size * 64 * 0.30103) + 32
        out = C.create_string_buffer(cap)
        n = C.c_size_t(0)
        rc = self.lib.ref_to_dec_string(_p64(leaves), leaves.size, out, cap, C.byref(n))
        if rc != 0:
            raise OracleError(f"ref_to_dec_string returned {rc}")
        return out.raw[: n.value].decode()

    def from_dec_string(self, text: bytes):
        """BigInt(text) (decimal): (Digits, negative)."""
        cap = len(text) // 8 + 8
        out = np.zeros(cap, dtype=np.uint32)
        n, neg = C.c_size_t(0), C.c_int(0)
        rc = self.lib.ref_from_dec_string(text, len(text), _p32(out), cap, C.byref(n), C.byref(neg))
        if rc != 0:
            raise OracleError(f"ref_from_dec_string returned {rc}")
        return out[: n.value].copy(), bool(neg.value)

    def fast_pow_digits(self, base: int, exponent: int) -> np.ndarray:
        """fast_pow(BigInt(base), exponent) as reference 28-bit Digits."""
        cap = (int(exponent) * 64) // 28 + 8
        out = np.zeros(cap, dtype=np.uint32)
        n = C.c_size_t(0)
        rc = self.lib.ref_fast_pow(int(base), int(exponent), _p32(out), cap, C.byref(n))
        if rc != 0:
            raise OracleError(f"ref_fast_pow returned {rc}")
        return out[: n.value].copy()

    def product_tree_digits(self, leaves) -> np.ndarray:
        leaves = _limbs(leaves)
        cap = (leaves.size * 64) // 28 + 8
        out = np.zeros(cap, dtype=np.uint32)
        n = C.c_size_t(0)
        rc = self.lib.ref_product_tree(_p64(leaves), leaves.size, _p32(out), cap, C.byref(n))
        if rc != 0:
            raise OracleError(f"ref_product_tree returned {rc}")
        return out[: n.value].copy()


def have_reference() -> bool:
    return os.path.exists(REF_SO)


def have_reference_gpu() -> bool:
    return os.path.exists(REF_GPU_SO)


def digits28_to_limbs(d) -> np.ndarray:
    """Pack little-endian 28-bit digits into u64 limbs (leading zeros stripped)."""
    d = _digits(d)
    v = 0
    for i in range(d.size - 1, -1, -1):
        v = (v << 28) | int(d[i])
    return int_to_limbs(v)


def int_to_limbs(v: int) -> np.ndarray:
    out = []
    while v:
        out.append(v & 0xFFFFFFFFFFFFFFFF)
        v >>= 64
    return np.array(out, dtype=np.uint64)


def limbs_to_int(x) -> int:
    x = _limbs(x)
    return int.from_bytes(x.astype("<u8").tobytes(), "little")
