"""C-ABI surface checks that need no GPU: the library loads, exports every
entry point declared in include/*.h, and rejects bad arguments on the host
before touching a device."""
from __future__ import annotations

import ctypes as C
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_recipe

LIB = os.path.join(ROOT, "bigint_b200", "libbigint_b200.so")


def declared_functions() -> list[str]:
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(bgpu_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    load_recipe("bigint_b200/build.py").build()
    import bigint_b200

    return bigint_b200.lib


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("bgpu_init", "bgpu_shutdown", "bgpu_strerror", "bgpu_mul_u64", "bgpu_mul_digits",
                 "bgpu_mul_u64_device", "bgpu_device_status", "bgpu_mul_u64_many", "bgpu_pow_u64",
                 "bgpu_reciprocal_digits", "bgpu_from_decimal", "bgpu_to_decimal", "bgpu_divmod_digits",
                 "bgpu_bigfloat_to_decimal"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT\s+(bgpu_\w+)", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        assert hasattr(lib, n)


def test_strerror(lib):
    assert lib.bgpu_strerror(0) == b"ok"
    assert b"output buffer" in lib.bgpu_strerror(-5)
    assert lib.bgpu_strerror(12345) == b"unknown status"


def test_invalid_arguments_rejected_on_host(lib):
    u64p = C.POINTER(C.c_uint64)
    n = C.c_size_t(0)
    a = np.ones(4, dtype=np.uint64)
    pa = a.ctypes.data_as(u64p)
    assert lib.bgpu_mul_u64(None, 4, pa, 4, pa, 8, C.byref(n), 0, None) == -1
    assert lib.bgpu_mul_u64(pa, 0, pa, 4, pa, 8, C.byref(n), 0, None) == -1
    assert lib.bgpu_mul_u64(pa, 4, pa, 4, pa, 8, None, 0, None) == -1
    assert lib.bgpu_mul_u64(pa, 4, pa, 4, pa, 8, C.byref(n), 7, None) == -1  # unknown method
    u32p = C.POINTER(C.c_uint32)
    d = np.ones(4, dtype=np.uint32)
    pd = d.ctypes.data_as(u32p)
    assert lib.bgpu_mul_digits(pd, 0, pd, 4, 0, None, pd, 8, C.byref(n), 0, None) == -1
    assert lib.bgpu_mul_u64_device(None, 1, None, 1, None, 0, None) == -1


def test_calls_before_init_report_not_initialized(lib):
    lib.bgpu_shutdown()
    u64p = C.POINTER(C.c_uint64)
    n = C.c_size_t(0)
    a = np.ones(4, dtype=np.uint64)
    out = np.zeros(8, dtype=np.uint64)
    pa = a.ctypes.data_as(u64p)
    assert lib.bgpu_mul_u64(pa, 4, pa, 4, out.ctypes.data_as(u64p), 8, C.byref(n), 0, None) == -8
    assert lib.bgpu_device_status(None) == -8
    u32p = C.POINTER(C.c_uint32)
    d = np.ones(4, dtype=np.uint32)
    pd = d.ctypes.data_as(u32p)
    pp, neg = C.c_int64(0), C.c_int(0)
    assert lib.bgpu_reciprocal_digits(pd, 4, 0, 0, 0, pd, 4, C.byref(n), C.byref(pp), C.byref(neg)) == -8
    assert lib.bgpu_from_decimal(b"12", 2, pd, 4, C.byref(n), C.byref(neg)) == -8
    buf = C.create_string_buffer(16)
    assert lib.bgpu_to_decimal(pd, 4, 0, buf, 16, C.byref(n)) == -8
    n2, neg2 = C.c_size_t(0), C.c_int(0)
    assert lib.bgpu_divmod_digits(pd, 4, 0, pd, 2, 0, 0, 1, pd, 4, C.byref(n), C.byref(neg), pd, 4,
                                  C.byref(n2), C.byref(neg2)) == -8
    assert lib.bgpu_bigfloat_to_decimal(pd, 4, 0, 0, 0, buf, 16, C.byref(n)) == -8


def test_new_entry_points_reject_bad_arguments_on_host(lib):
    u32p = C.POINTER(C.c_uint32)
    d = np.ones(4, dtype=np.uint32)
    pd = d.ctypes.data_as(u32p)
    n, pp, neg = C.c_size_t(0), C.c_int64(0), C.c_int(0)
    buf = C.create_string_buffer(16)
    assert lib.bgpu_reciprocal_digits(None, 4, 0, 0, 0, pd, 4, C.byref(n), C.byref(pp), C.byref(neg)) == -1
    assert lib.bgpu_reciprocal_digits(pd, 0, 0, 0, 0, pd, 4, C.byref(n), C.byref(pp), C.byref(neg)) == -1
    assert lib.bgpu_reciprocal_digits(pd, 4, 0, 0, 0, pd, 4, None, C.byref(pp), C.byref(neg)) == -1
    assert lib.bgpu_from_decimal(b"12", 2, pd, 4, None, C.byref(neg)) == -1
    assert lib.bgpu_to_decimal(None, 4, 0, buf, 16, C.byref(n)) == -1
    assert lib.bgpu_to_decimal(pd, 0, 0, buf, 16, C.byref(n)) == -1
    assert lib.bgpu_to_decimal(pd, 4, 0, buf, 16, None) == -1
    n2, neg2 = C.c_size_t(0), C.c_int(0)

    def divmod_rc(a=pd, na=4, b=pd, nb=2, mode=0, q=pd, qlen=C.byref(n), rlen=C.byref(n2)):
        return lib.bgpu_divmod_digits(a, na, 0, b, nb, 0, mode, 1, q, 4, qlen, C.byref(neg), pd, 4, rlen,
                                      C.byref(neg2))

    assert divmod_rc(a=None) == -1
    assert divmod_rc(nb=0) == -1
    assert divmod_rc(mode=256) == -1
    assert divmod_rc(qlen=None) == -1
    assert divmod_rc(rlen=None) == -1
    assert lib.bgpu_bigfloat_to_decimal(None, 4, 0, 0, 0, buf, 16, C.byref(n)) == -1
    assert lib.bgpu_bigfloat_to_decimal(pd, 0, 0, 0, 0, buf, 16, C.byref(n)) == -1
    assert lib.bgpu_bigfloat_to_decimal(pd, 4, 0, 0, 0, buf, 16, None) == -1


def test_point_positions_beyond_the_bound_rejected_on_host(lib):
    """|point_pos| above 2^40 would overflow 28 * point_pos: rejected with
    BGPU_ERR_CAPACITY before any device work (no init needed)."""
    u32p = C.POINTER(C.c_uint32)
    d = np.ones(4, dtype=np.uint32)
    pd = d.ctypes.data_as(u32p)
    n, pp, neg = C.c_size_t(0), C.c_int64(0), C.c_int(0)
    buf = C.create_string_buffer(16)
    for bad in ((1 << 40) + 1, -(1 << 40) - 1, (1 << 62), -(1 << 63)):
        assert lib.bgpu_bigfloat_to_decimal(pd, 4, bad, 0, 0, buf, 16, C.byref(n)) == -4
        assert lib.bgpu_reciprocal_digits(pd, 4, bad, 0, 0, pd, 4, C.byref(n), C.byref(pp),
                                          C.byref(neg)) == -4


def header_constants() -> dict[str, int]:
    """Every `#define BGPU_NAME <integer>[u]` of include/*.h."""
    out = {}
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        for name, val in re.findall(r"^#define\s+(BGPU_\w+)\s+(-?(?:0x[0-9A-Fa-f]+|\d+))u?\b", open(h).read(),
                                    flags=re.M):
            out[name] = int(val, 0)
    return out


def test_python_constants_match_the_header(lib):
    """The Python binding's flag, method, status and tuning constants are the
    header's values (the binding passes them straight through the C-ABI)."""
    import bigint_b200._lib as L

    consts = header_constants()
    for must in ("BGPU_METHOD_NTT", "BGPU_INDEPENDENT", "BGPU_BATCH_PER_CLASS", "BGPU_FFT_AVERAGE_BOUND",
                 "BGPU_ERR_CAPACITY", "BGPU_NOALLOC_MAX_LIMBS"):
        assert must in consts, must
    shared = [n for n in consts if hasattr(L, n)]
    assert "BGPU_BATCH_PER_CLASS" in shared and "BGPU_INDEPENDENT" in shared
    for n in shared:
        assert getattr(L, n) == consts[n], n
