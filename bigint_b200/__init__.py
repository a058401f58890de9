"""bigint_b200 -- B200-native big-integer multiplication.

Python mirror of the reference's multiply interface (Looading99/BigInt,
``include/bigint/mul.h``) over the C-ABI in ``include/bigint_b200.h``:

=====================  ==============================================  =========================
this package           reference                                       C-ABI
=====================  ==============================================  =========================
``mul(A, B)``          ``bigint::mul::_mul`` (mul.h:208-220)           ``bgpu_mul_u64``
``ntt_mul(A, B)``      ``bigint::mul::ntt::mul`` (ntt_multithread.cpp:444) ``bgpu_mul_u64`` + NTT
``brute_mul(A, B)``    ``bigint::mul::brute::mul`` (mul.h:82-102)      ``bgpu_mul_u64`` + schoolbook
``karatsuba_mul(A, B)`` (none: the reference has no Karatsuba)         ``bgpu_mul_u64`` + Karatsuba
``fft_mul(A, B)``      ``bigint::mul::fft::mul`` (fft.cpp:281)         ``bgpu_mul_u64`` + FFT
``mul_digits(a, b,``   ``bigint::mul::mul_digits`` (mul.h:223-318)     ``bgpu_mul_digits``
``  precision, pos)``
``fast_pow(base, e)``  ``fast_pow<BigInt>`` (bigint_base.h:60-69)      ``bgpu_pow_u64``
``reciprocal_digits``  ``BigFloat::reciprocal`` (bigint.cpp:1044-1071) ``bgpu_reciprocal_digits``
``divmod_digits``      ``BigInt::divmod`` (bigint.cpp:625-673)          ``bgpu_divmod_digits``
``from_decimal(text)`` ``BigInt(const std::string&)`` (bigint.cpp:25-124) ``bgpu_from_decimal``
``to_decimal(d, neg)`` ``BigInt::print`` (bigint.cpp:175-247)          ``bgpu_to_decimal``
``bigfloat_to_decimal`` ``BigFloat::print`` (bigint.cpp:972-1041)       ``bgpu_bigfloat_to_decimal``
``init(device)``       ``bigint::init_thread_pool`` (bigint.h:35-38)   ``bgpu_init``
=====================  ==============================================  =========================

Operands are little-endian ``numpy.uint64`` limb arrays (or 28-bit
``numpy.uint32`` Digits for ``mul_digits``).  Passing the same array object
for both operands squares, as the reference detects squaring by address.
All arithmetic runs in the CUDA library ``libbigint_b200.so``; there is no
CPU fallback, and importing raises if the library is missing.
"""
from __future__ import annotations

from ._lib import (  # noqa: F401
    BGPU_FFT_AVERAGE_BOUND,
    BGPU_INDEPENDENT,
    BGPU_BATCH_PER_CLASS,
    BGPU_METHOD_AUTO,
    BGPU_METHOD_FFT,
    BGPU_METHOD_KARATSUBA,
    BGPU_METHOD_NTT,
    BGPU_METHOD_SCHOOLBOOK,
    BGPU_TUNE_BATCH_KARATSUBA_MAX_LIMBS,
    BGPU_TUNE_BATCH_SCHOOLBOOK_MAX_LIMBS,
    BGPU_TUNE_FFT_MAX_LIMBS,
    BGPU_TUNE_FFT_MIN_LIMBS,
    BGPU_TUNE_KARATSUBA_MAX_LIMBS,
    BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS,
    ROUND_CEIL,
    ROUND_FLOOR,
    ROUND_HALF_UP,
    ROUND_TRUNCATE,
    BatchPlan,
    BigIntGPUError,
    bigfloat_to_decimal,
    Stats,
    brute_mul,
    device_status,
    divmod_digits,
    fft_mul,
    from_decimal,
    get_batch_split,
    get_split,
    get_tuning,
    init,
    karatsuba_mul,
    kernel_times,
    last_launch_count,
    lib,
    load_tuning,
    library_path,
    mul,
    mul_batch_device,
    mul_device,
    mul_digits,
    mul_many,
    ntt_mul,
    fast_pow,
    product_tree,
    product_tree_device,
    reciprocal_digits,
    set_batch_split,
    set_block_limbs,
    set_split,
    set_kernel_timing,
    set_tuning,
    shutdown,
    to_decimal,
)
