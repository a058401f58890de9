"""ctypes binding of libbigint_b200.so (see include/bigint_b200.h)."""
from __future__ import annotations

import ctypes as C
import os
import threading
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
library_path = os.environ.get("BIGINT_B200_LIB", os.path.join(_HERE, "libbigint_b200.so"))

BGPU_OK = 0
BGPU_METHOD_AUTO = 0
BGPU_METHOD_NTT = 1
BGPU_METHOD_SCHOOLBOOK = 2
BGPU_METHOD_FFT = 3
BGPU_METHOD_KARATSUBA = 4
BGPU_FFT_AVERAGE_BOUND = 0x10
BGPU_INDEPENDENT = 0x20  # mul_device: operands not written by work in flight on the stream
BGPU_BATCH_PER_CLASS = 0x40  # BatchPlan: every NTT class its own launches on parallel graph branches
BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS = 1
BGPU_TUNE_BATCH_SCHOOLBOOK_MAX_LIMBS = 2
BGPU_TUNE_FFT_MIN_LIMBS = 3
BGPU_TUNE_FFT_MAX_LIMBS = 4
BGPU_TUNE_KARATSUBA_MAX_LIMBS = 5
BGPU_TUNE_BATCH_KARATSUBA_MAX_LIMBS = 6
DEFAULT_TUNING = os.path.join(_HERE, "tuning_b200.txt")

ERRORS = {
    -1: "BGPU_ERR_INVALID_ARG",
    -2: "BGPU_ERR_NO_DEVICE",
    -3: "BGPU_ERR_OOM",
    -4: "BGPU_ERR_CAPACITY",
    -5: "BGPU_ERR_OUT_CAPACITY",
    -6: "BGPU_ERR_CUDA",
    -7: "BGPU_ERR_DEVICE_TIMEOUT",
    -8: "BGPU_ERR_NOT_INIT",
}


class BigIntGPUError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        name = ERRORS.get(code, str(code))
        super().__init__(f"{what}: {name} ({lib.bgpu_strerror(code).decode()})")


class _Stats(C.Structure):
    _fields_ = [
        ("method", C.c_int32),
        ("log2_points", C.c_uint32),
        ("max_round_err", C.c_double),
        ("fell_back", C.c_int32),
        ("device_ms", C.c_float),
        ("fft_bits", C.c_int32),
    ]


@dataclass
class Stats:
    method: int
    log2_points: int
    max_round_err: float
    fell_back: bool
    device_ms: float
    fft_bits: int


class HostProduct(C.Structure):
    _fields_ = [("a", C.c_void_p), ("na", C.c_size_t), ("b", C.c_void_p), ("nb", C.c_size_t),
                ("out", C.c_void_p), ("out_cap", C.c_size_t), ("out_len", C.POINTER(C.c_size_t))]


class Product(C.Structure):
    _fields_ = [("a", C.c_void_p), ("na", C.c_size_t), ("b", C.c_void_p), ("nb", C.c_size_t),
                ("out", C.c_void_p)]


def _load() -> C.CDLL:
    if not os.path.exists(library_path):
        raise ImportError(
            f"bigint_b200: CUDA library not found at {library_path}; build it with "
            "`python bigint_b200/build.py` (there is no CPU fallback)")
    L = C.CDLL(library_path)
    u64p, u32p, szp = C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), C.POINTER(C.c_size_t)
    L.bgpu_init.argtypes = [C.c_int]
    L.bgpu_init.restype = C.c_int
    L.bgpu_shutdown.argtypes = []
    L.bgpu_shutdown.restype = C.c_int
    L.bgpu_strerror.argtypes = [C.c_int]
    L.bgpu_strerror.restype = C.c_char_p
    L.bgpu_mul_u64.argtypes = [u64p, C.c_size_t, u64p, C.c_size_t, u64p, C.c_size_t, szp,
                               C.c_uint32, C.POINTER(_Stats)]
    L.bgpu_mul_u64.restype = C.c_int
    L.bgpu_mul_digits.argtypes = [u32p, C.c_size_t, u32p, C.c_size_t, C.c_size_t,
                                  C.POINTER(C.c_int64), u32p, C.c_size_t, szp, C.c_uint32,
                                  C.POINTER(_Stats)]
    L.bgpu_mul_digits.restype = C.c_int
    L.bgpu_selftest_wait.argtypes = [C.c_uint32, C.c_int]
    L.bgpu_selftest_wait.restype = C.c_int
    L.bgpu_mul_u64_many.argtypes = [C.POINTER(HostProduct), C.c_size_t, C.c_uint32]
    L.bgpu_mul_u64_many.restype = C.c_int
    L.bgpu_pow_u64.argtypes = [u64p, C.c_size_t, C.c_uint32, u64p, C.c_size_t, szp]
    L.bgpu_pow_u64.restype = C.c_int
    L.bgpu_to_decimal.argtypes = [u32p, C.c_size_t, C.c_int, C.c_char_p, C.c_size_t, szp]
    L.bgpu_to_decimal.restype = C.c_int
    L.bgpu_from_decimal.argtypes = [C.c_char_p, C.c_size_t, u32p, C.c_size_t, szp, C.POINTER(C.c_int)]
    L.bgpu_from_decimal.restype = C.c_int
    L.bgpu_reciprocal_digits.argtypes = [u32p, C.c_size_t, C.c_int64, C.c_int, C.c_size_t, u32p,
                                         C.c_size_t, szp, C.POINTER(C.c_int64), C.POINTER(C.c_int)]
    L.bgpu_reciprocal_digits.restype = C.c_int
    L.bgpu_divmod_digits.argtypes = [u32p, C.c_size_t, C.c_int, u32p, C.c_size_t, C.c_int, C.c_uint32, C.c_int,
                                     u32p, C.c_size_t, C.POINTER(C.c_size_t), C.POINTER(C.c_int), u32p,
                                     C.c_size_t, C.POINTER(C.c_size_t), C.POINTER(C.c_int)]
    L.bgpu_divmod_digits.restype = C.c_int
    L.bgpu_bigfloat_to_decimal.argtypes = [u32p, C.c_size_t, C.c_int64, C.c_int, C.c_size_t, C.c_char_p,
                                           C.c_size_t, C.POINTER(C.c_size_t)]
    L.bgpu_bigfloat_to_decimal.restype = C.c_int
    L.bgpu_set_block_limbs.argtypes = [C.c_uint64]
    L.bgpu_set_block_limbs.restype = C.c_int
    L.bgpu_mul_u64_device.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p,
                                      C.c_uint32, C.c_void_p]
    L.bgpu_mul_u64_device.restype = C.c_int
    L.bgpu_device_status.argtypes = [C.c_void_p]
    L.bgpu_device_status.restype = C.c_int
    L.bgpu_last_launch_count.argtypes = []
    L.bgpu_last_launch_count.restype = C.c_uint32
    L.bgpu_batch_plan_create.argtypes = [C.POINTER(Product), C.c_size_t, C.c_uint32,
                                         C.POINTER(C.c_void_p)]
    L.bgpu_batch_plan_create.restype = C.c_int
    L.bgpu_batch_plan_run.argtypes = [C.c_void_p, C.c_void_p]
    L.bgpu_batch_plan_run.restype = C.c_int
    L.bgpu_batch_plan_destroy.argtypes = [C.c_void_p]
    L.bgpu_batch_plan_destroy.restype = C.c_int
    L.bgpu_batch_plan_launches.argtypes = [C.c_void_p]
    L.bgpu_batch_plan_launches.restype = C.c_uint32
    L.bgpu_mul_batch_device.argtypes = [C.POINTER(Product), C.c_size_t, C.c_uint32, C.c_void_p]
    L.bgpu_mul_batch_device.restype = C.c_int
    L.bgpu_product_tree_device.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p]
    L.bgpu_product_tree_device.restype = C.c_int
    L.bgpu_product_tree_u64.argtypes = [u64p, C.c_size_t, u64p, C.c_size_t, szp]
    L.bgpu_product_tree_u64.restype = C.c_int
    L.bgpu_set_split.argtypes = [C.c_uint32, C.c_uint32]
    L.bgpu_set_split.restype = C.c_int
    L.bgpu_get_split.argtypes = [C.c_uint32]
    L.bgpu_get_split.restype = C.c_int
    L.bgpu_set_batch_split.argtypes = [C.c_uint32, C.c_uint32]
    L.bgpu_set_batch_split.restype = C.c_int
    L.bgpu_get_batch_split.argtypes = [C.c_uint32]
    L.bgpu_get_batch_split.restype = C.c_int
    L.bgpu_set_tuning.argtypes = [C.c_uint32, C.c_uint64]
    L.bgpu_set_tuning.restype = C.c_int
    L.bgpu_get_tuning.argtypes = [C.c_uint32, C.POINTER(C.c_uint64)]
    L.bgpu_get_tuning.restype = C.c_int
    L.bgpu_load_tuning.argtypes = [C.c_char_p]
    L.bgpu_load_tuning.restype = C.c_int
    L.bgpu_set_kernel_timing.argtypes = [C.c_int]
    L.bgpu_set_kernel_timing.restype = C.c_int
    L.bgpu_kernel_times.argtypes = [C.POINTER(C.c_char_p), C.POINTER(C.c_float), C.c_int,
                                    C.POINTER(C.c_uint32)]
    L.bgpu_kernel_times.restype = C.c_int
    return L


lib = _load()
_init_lock = threading.Lock()
_initialized_device: int | None = None


def _check(rc: int, what: str) -> None:
    if rc != BGPU_OK:
        raise BigIntGPUError(rc, what)


def init(device: int = 0) -> None:
    """Select the CUDA device and build the twiddle tables (idempotent).

    On first use applies a tuning table: the one named by the environment
    variable BIGINT_B200_TUNING, else the autotuner's table shipped with the
    package (``tuning_b200.txt``, measured on a B200) when the device is a
    B200; BIGINT_B200_TUNING set to the empty string keeps the built-in
    choices."""
    global _initialized_device
    with _init_lock:
        first = _initialized_device is None
        _check(lib.bgpu_init(int(device)), "bgpu_init")
        _initialized_device = int(device)
        if first:
            path = os.environ.get("BIGINT_B200_TUNING")
            if path is None and os.path.exists(DEFAULT_TUNING) and _device_is_b200():
                path = DEFAULT_TUNING
            if path:
                load_tuning(path)


def _device_is_b200() -> bool:
    try:
        import torch

        return "B200" in torch.cuda.get_device_name(_initialized_device or 0)
    except Exception:
        return False


def load_tuning(path: str) -> None:
    """Apply a tuning table written by ``bigint_b200.autotune`` (bgpu_load_tuning)."""
    _check(lib.bgpu_load_tuning(os.fsencode(path)), f"bgpu_load_tuning({path})")


def set_tuning(key: int, value: int) -> None:
    _check(lib.bgpu_set_tuning(int(key), int(value)), "bgpu_set_tuning")


def get_tuning(key: int) -> int:
    v = C.c_uint64(0)
    _check(lib.bgpu_get_tuning(int(key), C.byref(v)), "bgpu_get_tuning")
    return int(v.value)


def shutdown() -> None:
    global _initialized_device
    with _init_lock:
        lib.bgpu_shutdown()
        _initialized_device = None


def _ensure_init() -> None:
    if _initialized_device is None:
        init(int(os.environ.get("BIGINT_B200_DEVICE", "0")))


def _as_limbs(x) -> np.ndarray:
    a = np.asarray(x)
    if a.dtype != np.uint64:
        a = a.astype(np.uint64)
    return np.ascontiguousarray(a)


def _as_digits(x) -> np.ndarray:
    a = np.asarray(x)
    if a.dtype != np.uint32:
        a = a.astype(np.uint32)
    return np.ascontiguousarray(a)


def _stats(s: _Stats) -> Stats:
    return Stats(int(s.method), int(s.log2_points), float(s.max_round_err), bool(s.fell_back),
                 float(s.device_ms), int(s.fft_bits))


def _mul_u64(A, B, flags: int, stats: bool, out=None):
    _ensure_init()
    square = B is None or B is A
    a = _as_limbs(A)
    b = a if square else _as_limbs(B)
    if a.size == 0 or b.size == 0:
        raise BigIntGPUError(-1, "bgpu_mul_u64 (empty operand)")
    if out is None:
        out = np.empty(a.size + b.size, dtype=np.uint64)
    elif out.dtype != np.uint64 or not out.flags.c_contiguous:
        raise ValueError("out must be a contiguous uint64 array")
    n = C.c_size_t(0)
    st = _Stats()
    u64p = C.POINTER(C.c_uint64)
    pa = a.ctypes.data_as(u64p)
    pb = pa if square else b.ctypes.data_as(u64p)
    rc = lib.bgpu_mul_u64(pa, a.size, pb, b.size, out.ctypes.data_as(u64p), out.size,
                          C.byref(n), flags, C.byref(st))
    _check(rc, "bgpu_mul_u64")
    res = out[: n.value]
    return (res, _stats(st)) if stats else res


def mul(A, B=None, *, stats: bool = False, out=None):
    """A*B for little-endian u64 limb arrays (``_mul``, mul.h:208-220).

    ``mul(A)`` or ``mul(A, A)`` squares.  Returns the product without leading
    zero limbs (an empty array for a zero operand).  ``out`` may supply the
    destination (e.g. pinned host memory); the result is a view of it."""
    return _mul_u64(A, B, BGPU_METHOD_AUTO, stats, out)


def mul_many(pairs, outs=None, method: int = BGPU_METHOD_AUTO) -> list:
    """Products of many host-resident pairs in one pipelined call
    (``bgpu_mul_u64_many``): copies of neighbouring products overlap the
    multiplies.  ``pairs`` is a list of (A, B) limb arrays (B None or A
    itself squares); ``outs`` optionally gives each destination (>= na + nb
    limbs, page-locked for overlap).  Returns the products as views without
    leading zeros."""
    _ensure_init()
    n = len(pairs)
    arr = (HostProduct * max(1, n))()
    lens = (C.c_size_t * max(1, n))()
    keep, res = [], []
    for i, (A, B) in enumerate(pairs):
        a = _as_limbs(A)
        b = a if (B is None or B is A) else _as_limbs(B)
        if a.size == 0 or b.size == 0:
            raise BigIntGPUError(-1, "bgpu_mul_u64_many (empty operand)")
        o = outs[i] if outs is not None else np.empty(a.size + b.size, dtype=np.uint64)
        if o.dtype != np.uint64 or not o.flags.c_contiguous or o.size < a.size + b.size:
            raise ValueError("each out must be a contiguous uint64 array of >= na + nb limbs")
        keep += [a, b, o]
        res.append(o)
        len_ptr = C.cast(C.addressof(lens) + i * C.sizeof(C.c_size_t), C.POINTER(C.c_size_t))
        arr[i] = HostProduct(a.ctypes.data, a.size, b.ctypes.data, b.size, o.ctypes.data, o.size, len_ptr)
    _check(lib.bgpu_mul_u64_many(arr, n, method), "bgpu_mul_u64_many")
    return [res[i][: lens[i]] for i in range(n)]


def ntt_mul(A, B=None, *, stats: bool = False):
    """A*B forced onto the three-prime NTT (``ntt::mul``, ntt_multithread.cpp:444)."""
    return _mul_u64(A, B, BGPU_METHOD_NTT, stats)


def brute_mul(A, B=None, *, stats: bool = False):
    """A*B on the schoolbook kernel (``brute::mul``, mul.h:82-102); na+nb <= 256."""
    return _mul_u64(A, B, BGPU_METHOD_SCHOOLBOOK, stats)


def karatsuba_mul(A, B=None, *, stats: bool = False):
    """A*B on the Karatsuba kernel (one level over column sums); na, nb <= 256.
    The reference has no Karatsuba: its small products use brute::mul."""
    return _mul_u64(A, B, BGPU_METHOD_KARATSUBA, stats)


def fft_mul(A, B=None, *, digit_bits: int = 0, average_bound: bool = False, stats: bool = False):
    """A*B through the FP64 complex-FFT form (``fft::mul``, fft.cpp:281).

    ``digit_bits`` forces the bits per point (8..20; 0 = from the error
    bound).  The result is exact: a product whose max rounding distance
    exceeds 1/4 is recomputed on the NTT (reported in ``stats``)."""
    flags = BGPU_METHOD_FFT | (int(digit_bits) << 8) | (BGPU_FFT_AVERAGE_BOUND if average_bound else 0)
    return _mul_u64(A, B, flags, stats)


def fast_pow(base, exponent: int) -> np.ndarray:
    """base**exponent (``fast_pow``, include/bigint/bigint_base.h:60-69) with
    every product of the squaring chain on the GPU.  ``base`` is a Python int
    >= 0 or a u64 limb array; returns little-endian u64 limbs."""
    _ensure_init()
    if isinstance(base, (int, np.integer)):
        v = int(base)
        if v < 0:
            raise ValueError("base must be non-negative")
        limbs = []
        while v:
            limbs.append(v & 0xFFFFFFFFFFFFFFFF)
            v >>= 64
        a = np.array(limbs or [0], dtype=np.uint64)
    else:
        a = _as_limbs(base)
    e = int(exponent)
    if not 0 <= e < 2**32:
        raise ValueError("exponent must fit in 32 bits (the reference's uint32_t)")
    bits = max(1, int(a.size) * 64)
    cap = max(1, (bits * max(e, 1) + 63) // 64 + 1)
    out = np.empty(cap, dtype=np.uint64)
    n = C.c_size_t(0)
    u64p = C.POINTER(C.c_uint64)
    _check(lib.bgpu_pow_u64(a.ctypes.data_as(u64p), a.size, e, out.ctypes.data_as(u64p), cap,
                            C.byref(n)), "bgpu_pow_u64")
    return out[: n.value]


def mul_digits(a, b=None, output_precision: int = 0, point_pos: int | None = None, *,
               method: int = BGPU_METHOD_AUTO, stats: bool = False):
    """Product of 28-bit Digits with the reference's ``mul_digits`` semantics.

    With ``point_pos`` given, returns ``(digits, new_point_pos)``."""
    _ensure_init()
    square = b is None or b is a
    da = _as_digits(a)
    db = da if square else _as_digits(b)
    if da.size == 0 or db.size == 0:
        raise BigIntGPUError(-1, "bgpu_mul_digits (empty operand)")
    cap = da.size + db.size + 2
    out = np.empty(cap, dtype=np.uint32)
    n = C.c_size_t(0)
    pp = C.c_int64(0 if point_pos is None else int(point_pos))
    st = _Stats()
    u32p = C.POINTER(C.c_uint32)
    pa = da.ctypes.data_as(u32p)
    pb = pa if square else db.ctypes.data_as(u32p)
    rc = lib.bgpu_mul_digits(pa, da.size, pb, db.size, int(output_precision),
                             C.byref(pp) if point_pos is not None else None,
                             out.ctypes.data_as(u32p), cap, C.byref(n), method, C.byref(st))
    _check(rc, "bgpu_mul_digits")
    res = out[: n.value]
    ret = (res, int(pp.value)) if point_pos is not None else res
    if stats:
        return ret, _stats(st)
    return ret


def to_decimal(digits, neg: bool = False) -> str:
    """Decimal text of a BigInt given by its 28-bit Digits and sign, as the
    reference's ``BigInt::print`` writes it (src/bigint.cpp:175-247); the
    conversion runs on the GPU (``bgpu_to_decimal``)."""
    _ensure_init()
    d = _as_digits(digits)
    if d.size == 0:
        raise BigIntGPUError(-1, "bgpu_to_decimal (empty input)")
    cap = int(d.size * 28 * 0.30103) + 64
    out = C.create_string_buffer(cap)
    n = C.c_size_t(0)
    _check(lib.bgpu_to_decimal(d.ctypes.data_as(C.POINTER(C.c_uint32)), d.size, int(bool(neg)), out, cap,
                               C.byref(n)), "bgpu_to_decimal")
    return out.raw[: n.value].decode()


def from_decimal(text):
    """Decimal text to ``(Digits, negative)``, as the reference's
    ``BigInt(const std::string&)`` reads it (src/bigint.cpp:25-124): a '-'
    before the first digit makes it negative, other non-digits are skipped.
    The value is built on the GPU (``bgpu_from_decimal``)."""
    _ensure_init()
    b = text.encode() if isinstance(text, str) else bytes(text)
    cap = len(b) // 8 + 8
    out = np.empty(cap, dtype=np.uint32)
    n, neg = C.c_size_t(0), C.c_int(0)
    _check(lib.bgpu_from_decimal(b, len(b), out.ctypes.data_as(C.POINTER(C.c_uint32)), cap, C.byref(n),
                                 C.byref(neg)), "bgpu_from_decimal")
    return out[: n.value], bool(neg.value)


def reciprocal_digits(digits, point_pos: int = 0, neg: bool = False, precision: int = 0):
    """``BigFloat::reciprocal(precision)`` (src/bigint.cpp:1044-1071) on the GPU.

    The input is a BigFloat's fields: 28-bit Digits without a leading zero
    digit, the point position (value = digits * 2^(-28 point_pos)) and the
    sign.  Returns ``(digits, point_pos, neg)`` of the reciprocal, identical to
    the reference's.  Every step of the Newton iteration keeps its digits on
    the device (``bgpu_reciprocal_digits``)."""
    _ensure_init()
    d = _as_digits(digits)
    if d.size == 0:
        raise BigIntGPUError(-1, "bgpu_reciprocal_digits (empty input)")
    u32p = C.POINTER(C.c_uint32)
    cap = 4 * max(int(precision), d.size) + 64
    for _ in range(2):
        out = np.empty(cap, dtype=np.uint32)
        n, pp, ng = C.c_size_t(0), C.c_int64(0), C.c_int(0)
        rc = lib.bgpu_reciprocal_digits(d.ctypes.data_as(u32p), d.size, int(point_pos), int(bool(neg)),
                                        int(precision), out.ctypes.data_as(u32p), cap, C.byref(n),
                                        C.byref(pp), C.byref(ng))
        if rc != -5:
            break
        cap = n.value
    _check(rc, "bgpu_reciprocal_digits")
    return out[: n.value], int(pp.value), bool(ng.value)


def bigfloat_to_decimal(digits, point_pos: int = 0, neg: bool = False, dec_digits: int = 0) -> str:
    """``BigFloat::print(out, dec_digits)`` (src/bigint.cpp:972-1041) on the GPU.

    The input is a BigFloat's fields: 28-bit Digits without a leading zero
    digit, the point position (value = digits * 2^(-28 point_pos)) and the
    sign.  Returns the reference's text, "[-]int.frac" with the fraction
    rounded half up to ``dec_digits`` digits (0: as many as its Digits hold)
    (``bgpu_bigfloat_to_decimal``)."""
    _ensure_init()
    d = _as_digits(digits)
    if d.size == 0:
        raise BigIntGPUError(-1, "bgpu_bigfloat_to_decimal (empty input)")
    u32p = C.POINTER(C.c_uint32)
    cap = int(d.size * 28 * 0.30103) + abs(int(point_pos)) * 9 + int(dec_digits) + 64
    for _ in range(2):
        out = C.create_string_buffer(cap)
        n = C.c_size_t(0)
        rc = lib.bgpu_bigfloat_to_decimal(d.ctypes.data_as(u32p), d.size, int(point_pos), int(bool(neg)),
                                          int(dec_digits), out, cap, C.byref(n))
        if rc != -5:
            break
        cap = n.value
    _check(rc, "bgpu_bigfloat_to_decimal")
    return out.raw[: n.value].decode()


ROUND_TRUNCATE, ROUND_FLOOR, ROUND_CEIL, ROUND_HALF_UP = 0, 1, 2, 3  # the reference's RoundMode


def divmod_digits(a, b, a_neg: bool = False, b_neg: bool = False, mode: int = ROUND_TRUNCATE,
                  check: bool = True):
    """``BigInt::divmod(b, mode, check)`` (src/bigint.cpp:625-673) on the GPU.

    ``a`` and ``b`` are 28-bit Digits without leading zeros (zero is ``[0]``)
    with separate signs.  Returns ``((q_digits, q_neg), (r_digits, r_neg))``,
    identical to the reference's quotient and remainder; the reciprocal, the
    estimate, Q * b and the adjustment all run on the device
    (``bgpu_divmod_digits``)."""
    _ensure_init()
    da, db = _as_digits(a), _as_digits(b)
    if da.size == 0 or db.size == 0:
        raise BigIntGPUError(-1, "bgpu_divmod_digits (empty input)")
    u32p = C.POINTER(C.c_uint32)
    qcap, rcap = max(da.size - db.size + 2, 1), max(db.size, 1) + 1
    for _ in range(2):
        q, r = np.empty(qcap, dtype=np.uint32), np.empty(rcap, dtype=np.uint32)
        nq, nr, qn, rn = C.c_size_t(0), C.c_size_t(0), C.c_int(0), C.c_int(0)
        rc = lib.bgpu_divmod_digits(da.ctypes.data_as(u32p), da.size, int(bool(a_neg)), db.ctypes.data_as(u32p),
                                    db.size, int(bool(b_neg)), int(mode), int(bool(check)),
                                    q.ctypes.data_as(u32p), qcap, C.byref(nq), C.byref(qn),
                                    r.ctypes.data_as(u32p), rcap, C.byref(nr), C.byref(rn))
        if rc != -5:
            break
        qcap, rcap = max(qcap, nq.value), max(rcap, nr.value)
    _check(rc, "bgpu_divmod_digits")
    return (q[: nq.value], bool(qn.value)), (r[: nr.value], bool(rn.value))


def mul_device(a_ptr: int, na: int, b_ptr: int, nb: int, out_ptr: int, stream: int = 0,
               method: int = BGPU_METHOD_AUTO) -> None:
    """Asynchronous product of device-resident limbs (``bgpu_mul_u64_device``).

    ``out_ptr`` receives na+nb limbs.  Equal pointers and lengths square.
    ``stream`` is a cudaStream_t handle (0 = legacy default stream), e.g.
    ``torch.cuda.current_stream().cuda_stream``.  ``method`` may include
    ``BGPU_INDEPENDENT`` for a stream of independent products (the next
    product's transform starts under the previous one's carry scan)."""
    _ensure_init()
    rc = lib.bgpu_mul_u64_device(C.c_void_p(a_ptr), na, C.c_void_p(b_ptr), nb,
                                 C.c_void_p(out_ptr), method, C.c_void_p(stream or None))
    _check(rc, "bgpu_mul_u64_device")


def device_status(stream: int = 0) -> None:
    """Synchronize ``stream`` and raise if a device-side error was recorded."""
    _check(lib.bgpu_device_status(C.c_void_p(stream or None)), "bgpu_device_status")


def last_launch_count() -> int:
    return int(lib.bgpu_last_launch_count())


def set_block_limbs(limbs: int) -> None:
    """Operand block of the products beyond the largest transform (a power of
    two in [64, 2^24] limbs; 0 = the default 2^24).  A test hook: with a small
    block, products above 4 * limbs points take the block path."""
    _check(lib.bgpu_set_block_limbs(int(limbs)), "bgpu_set_block_limbs")


def set_split(log2_points: int, log2_column: int) -> None:
    """Column-pass length 2^log2_column for 2^log2_points-point transforms (0 = default)."""
    _check(lib.bgpu_set_split(int(log2_points), int(log2_column)), "bgpu_set_split")


def set_batch_split(log2_points: int, log2_column: int) -> None:
    """Column-pass length for the NTT classes of batch plans and product trees."""
    _check(lib.bgpu_set_batch_split(int(log2_points), int(log2_column)), "bgpu_set_batch_split")


def get_batch_split(log2_points: int) -> int:
    r = lib.bgpu_get_batch_split(int(log2_points))
    if r < 0:
        _check(r, "bgpu_get_batch_split")
    return r


def get_split(log2_points: int) -> int:
    r = lib.bgpu_get_split(int(log2_points))
    if r < 0:
        _check(r, "bgpu_get_split")
    return r


def set_kernel_timing(on: bool) -> None:
    """Record CUDA events between the kernels of each NTT product."""
    _ensure_init()
    _check(lib.bgpu_set_kernel_timing(int(bool(on))), "bgpu_set_kernel_timing")


def kernel_times() -> tuple[list[tuple[str, float]], int]:
    """Mean (kernel name, ms) over the NTT products timed since
    ``set_kernel_timing(True)``, in launch order, and the product count."""
    names = (C.c_char_p * 8)()
    ms = (C.c_float * 8)()
    cnt = C.c_uint32(0)
    n = lib.bgpu_kernel_times(names, ms, 8, C.byref(cnt))
    if n < 0:
        _check(n, "bgpu_kernel_times")
    return [(names[i].decode(), float(ms[i])) for i in range(n)], int(cnt.value)


class BatchPlan:
    """A batch of independent device-resident products, captured in one CUDA
    graph (``bgpu_batch_plan_*``).  ``products`` is a list of
    ``(a_ptr, na, b_ptr, nb, out_ptr)`` device pointers/lengths."""

    def __init__(self, products, flags: int = 0):
        _ensure_init()
        arr = (Product * max(1, len(products)))()
        for i, (a, na, b, nb, out) in enumerate(products):
            arr[i] = Product(C.c_void_p(a), na, C.c_void_p(b), nb, C.c_void_p(out))
        self._h = C.c_void_p()
        _check(lib.bgpu_batch_plan_create(arr, len(products), flags, C.byref(self._h)),
               "bgpu_batch_plan_create")
        self.count = len(products)

    @property
    def launches(self) -> int:
        return int(lib.bgpu_batch_plan_launches(self._h))

    def run(self, stream: int = 0) -> None:
        _check(lib.bgpu_batch_plan_run(self._h, C.c_void_p(stream or None)), "bgpu_batch_plan_run")

    def close(self) -> None:
        if self._h:
            lib.bgpu_batch_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mul_batch_device(products, stream: int = 0, flags: int = 0) -> None:
    """One-shot batch (create, run, synchronize, destroy)."""
    _ensure_init()
    arr = (Product * max(1, len(products)))()
    for i, (a, na, b, nb, out) in enumerate(products):
        arr[i] = Product(C.c_void_p(a), na, C.c_void_p(b), nb, C.c_void_p(out))
    _check(lib.bgpu_mul_batch_device(arr, len(products), flags, C.c_void_p(stream or None)),
           "bgpu_mul_batch_device")


def product_tree(leaves) -> np.ndarray:
    """Pairwise product tree of u64 values (binary splitting, examples/pi.cpp:41-80)."""
    _ensure_init()
    x = _as_limbs(leaves)
    if x.size == 0:
        raise BigIntGPUError(-1, "bgpu_product_tree_u64 (no leaves)")
    width = 1 << max(0, (x.size - 1).bit_length())
    out = np.empty(width, dtype=np.uint64)
    n = C.c_size_t(0)
    u64p = C.POINTER(C.c_uint64)
    _check(lib.bgpu_product_tree_u64(x.ctypes.data_as(u64p), x.size, out.ctypes.data_as(u64p),
                                     out.size, C.byref(n)), "bgpu_product_tree_u64")
    return out[: n.value]


def product_tree_device(leaves_ptr: int, n: int, out_ptr: int, out_cap: int, stream: int = 0) -> None:
    """Device-resident product tree; out receives the power-of-two width >= n limbs."""
    _ensure_init()
    _check(lib.bgpu_product_tree_device(C.c_void_p(leaves_ptr), n, C.c_void_p(out_ptr), out_cap,
                                        C.c_void_p(stream or None)), "bgpu_product_tree_device")
