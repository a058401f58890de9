"""The FP64 complex-FFT form (fft::mul, src/mul/fft.cpp:281-384) on the GPU:
every product must come out exact -- either the FFT's rounding distance
stays within 1/4 or the product is recomputed on the NTT -- and the recorded
error statistics must behave as the error bound says."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED, golden_u64_cases, rand_limbs
from oracle.pyoracle import limbs_to_int

pytestmark = pytest.mark.gpu
ONES = np.uint64(0xFFFFFFFFFFFFFFFF)


def test_golden_through_fft(bb, golden):
    for kind, a, b, c in golden_u64_cases(golden):
        args = (a,) if b is None else (a, b)
        got, st = bb.fft_mul(*args, stats=True)
        assert np.array_equal(got, c), (kind, a.size)
        if st.method == bb.BGPU_METHOD_FFT:
            assert st.max_round_err < 0.25 and not st.fell_back, (kind, st)


@pytest.mark.parametrize("n", [1000, 20000, 1 << 16, 1 << 18])
def test_worst_case_bound_random_never_falls_back(bb, port, n):
    rng = np.random.default_rng(SEED + n)
    a, b = rand_limbs(rng, n), rand_limbs(rng, n)
    got, st = bb.fft_mul(a, b, stats=True)
    assert st.method == bb.BGPU_METHOD_FFT and not st.fell_back
    assert 0.0 <= st.max_round_err < 0.25
    assert np.array_equal(got, port.mul(a, b))


@pytest.mark.parametrize("n", [4096, 1 << 16, 1 << 18])
def test_worst_case_bound_all_ones(bb, port, n):
    ones = np.full(n, ONES)
    got, st = bb.fft_mul(ones, stats=True)
    assert st.method == bb.BGPU_METHOD_FFT and not st.fell_back and st.max_round_err < 0.25
    assert np.array_equal(got, port.ntt_mul(ones))


def test_average_bound_uses_more_bits_and_stays_exact(bb, port):
    rng = np.random.default_rng(SEED + 21)
    n = 1 << 16
    a, b = rand_limbs(rng, n), rand_limbs(rng, n)
    _, st_w = bb.fft_mul(a, b, stats=True)
    got, st_a = bb.fft_mul(a, b, average_bound=True, stats=True)
    assert st_a.fft_bits > st_w.fft_bits
    assert np.array_equal(got, port.mul(a, b))


def test_oversized_points_fall_back_to_ntt(bb, port):
    """20-bit points on all-ones operands of 2^18 limbs: coefficients near
    2^58 cannot be represented in FP64, the error check trips and the NTT
    recomputes the product, so the result is still exact."""
    ones = np.full(1 << 18, ONES)
    got, st = bb.fft_mul(ones, digit_bits=20, stats=True)
    assert st.fell_back and st.max_round_err > 0.25
    assert np.array_equal(got, port.ntt_mul(ones))


@pytest.mark.parametrize("bits", range(8, 21))
def test_forced_bits_small(bb, bits):
    """Forced b = 8..20 at small sizes (the reference's forced-B regression,
    tests/measure_digit_bits.cpp:186-201)."""
    rng = np.random.default_rng(SEED + 100 + bits)
    for _ in range(3):
        a, b = rand_limbs(rng, 40), rand_limbs(rng, 31)
        got, st = bb.fft_mul(a, b, digit_bits=bits, stats=True)
        assert st.fft_bits == bits
        assert limbs_to_int(got) == limbs_to_int(a) * limbs_to_int(b)


def test_fft_square_and_unbalanced(bb, port):
    rng = np.random.default_rng(SEED + 22)
    a = rand_limbs(rng, 30000)
    assert np.array_equal(bb.fft_mul(a), port.ntt_mul(a))
    b = rand_limbs(rng, 300)
    assert np.array_equal(bb.fft_mul(a, b), port.mul(a, b))


def test_reference_regression_sizes(bb, port):
    """The reference's own FFT regression (tests/measure_digit_bits.cpp:135-168):
    uniform 28-bit digits at {200, 500, 1000, 3000, 8000, 20000, 25000}
    digits, four repetitions each, automatic bits per point, against the
    integer product."""
    from oracle.pyoracle import digits28_to_limbs

    rng = np.random.default_rng(SEED)
    for nd in (200, 500, 1000, 3000, 8000, 20000, 25000):
        for _ in range(4):
            a = rng.integers(0, 1 << 28, nd, dtype=np.uint32)
            b = rng.integers(0, 1 << 28, nd, dtype=np.uint32)
            a[-1] |= 1
            b[-1] |= 1
            la, lb = digits28_to_limbs(a), digits28_to_limbs(b)
            got, st = bb.fft_mul(la, lb, stats=True)
            assert np.array_equal(got, port.mul(la, lb)), nd
            assert st.method == bb.BGPU_METHOD_FFT and st.max_round_err < 0.25, (nd, st)


def test_smallest_transforms(bb):
    """Products of one to a few limbs through the FFT form: the shortest
    transforms (the reference's radix-4 FFT mishandles length 4,
    src/mul/fft.cpp:135; nothing here may)."""
    rng = np.random.default_rng(SEED + 23)
    for na, nb in [(1, 1), (1, 2), (2, 2), (3, 1), (4, 4), (5, 3)]:
        for fill in ("rand", "ones"):
            a = np.full(na, ONES) if fill == "ones" else rand_limbs(rng, na)
            b = np.full(nb, ONES) if fill == "ones" else rand_limbs(rng, nb)
            got = bb.fft_mul(a, b)
            assert limbs_to_int(got) == limbs_to_int(a) * limbs_to_int(b), (na, nb, fill)


@pytest.mark.parametrize("n,average,log_points", [(1 << 20, False, 24), ((1 << 20) + 1000, False, 25),
                                                  (1 << 20, True, 24), (1 << 22, True, 26)])
def test_large_transforms_exact_vs_ntt(bb, n, average, log_points):
    """The transforms beyond 2^23 complex points (2^11- to 2^13-row column
    tiles of 4, 2 and 1 columns): 2^26- and 2^28-bit operands, exact whether
    or not the product falls back to the NTT, with the expected length."""
    rng = np.random.default_rng(SEED + n + average)
    a, b = rand_limbs(rng, n), rand_limbs(rng, n)
    got, st = bb.fft_mul(a, b, average_bound=average, stats=True)
    assert st.method == bb.BGPU_METHOD_FFT and st.log2_points == log_points, st
    assert np.array_equal(got, bb.ntt_mul(a, b))
    if not average:
        assert not st.fell_back and st.max_round_err < 0.25


def test_large_transform_all_ones_square(bb):
    ones = np.full(1 << 20, ONES)
    got, st = bb.fft_mul(ones, stats=True)
    assert st.method == bb.BGPU_METHOD_FFT and st.log2_points == 24 and not st.fell_back
    assert np.array_equal(got, bb.ntt_mul(ones))
