"""Products beyond the largest transform (2^26 points, 2^31 product bits).

The reference switches to Schoenhage-Strassen there (src/mul/ssa.cpp:383);
the engine cuts both operands into 2^30-bit blocks, transforms every block
once, forms each output block's sum of block products in the transform
domain (at most as many products per sum as the CRT modulus allows: two at
this block size), inverse-transforms each sum and adds it into the result
with a device carry scan.  At these sizes the CPU oracle takes minutes, so
the checks are size-independent: the residue identity mod 2^61-1, the low
limb, operand order, and the all-ones closed form, whose carries cross every
block boundary and whose coefficients are the largest the bound admits.  The
block path is also run with small blocks (the bgpu_set_block_limbs test hook)
and compared limb-exact with the oracle, with 2^22-limb blocks on the strict
prime set against one whole transform, and with rows too short for the
spectral row passes, where every block pair is one NTT product."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED, rand_digits, rand_limbs

pytestmark = pytest.mark.gpu
M61 = (1 << 61) - 1
ONES = np.uint64(0xFFFFFFFFFFFFFFFF)
BLOCK = 1 << 24  # limbs per operand block


def check_product(port, a, b, c):
    assert c.size == a.size + b.size
    assert port.mod_m61(a) * port.mod_m61(b) % M61 == port.mod_m61(c)
    assert (int(a[0]) * int(b[0])) & ((1 << 64) - 1) == int(c[0])


def test_general_2p31_product(bb, port):
    """2^31 x 2^31 bits: two blocks each, three spectral sums (the middle one
    of two block products)."""
    rng = np.random.default_rng(SEED + 500)
    n = 2 * BLOCK
    a, b = rand_limbs(rng, n), rand_limbs(rng, n)
    c, st = bb.mul(a, b, stats=True)
    check_product(port, a, b, c)
    assert np.array_equal(bb.mul(b, a), c)


def test_uneven_blocks_and_ragged_tails(bb, port):
    rng = np.random.default_rng(SEED + 501)
    a, b = rand_limbs(rng, 3 * BLOCK + 5), rand_limbs(rng, BLOCK + 77)
    c = bb.mul(a, b)
    check_product(port, a, b, c)
    assert np.array_equal(bb.mul(b, a), c)


def test_all_ones_square_crosses_blocks(bb):
    """(2^k - 1)^2 = 2^2k - 2^(k+1) + 1: every block product's carry runs
    through the all-ones limbs of the result."""
    n = 2 * BLOCK + 3
    ones = np.full(n, ONES)
    c = bb.mul(ones)
    assert c.size == 2 * n
    assert c[0] == 1 and not c[1:n].any() and c[n] == np.uint64(0xFFFFFFFFFFFFFFFE)
    assert np.all(c[n + 1:] == ONES)
    c2 = bb.mul(ones, ones.copy())  # distinct buffers: the general path
    assert np.array_equal(c2, c)


def test_square_matches_general(bb, port):
    rng = np.random.default_rng(SEED + 502)
    a = rand_limbs(rng, 2 * BLOCK + 1000)
    sq = bb.mul(a)
    assert np.array_equal(sq, bb.mul(a, a.copy()))
    ra = port.mod_m61(a)
    assert ra * ra % M61 == port.mod_m61(sq)


def test_device_entry(bb, port):
    import torch

    rng = np.random.default_rng(SEED + 503)
    a, b = rand_limbs(rng, BLOCK + 12345), rand_limbs(rng, BLOCK + 999)
    dev = torch.device("cuda", 0)
    da = torch.from_numpy(a.view(np.int64)).to(dev)
    db = torch.from_numpy(b.view(np.int64)).to(dev)
    out = torch.empty(a.size + b.size, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()
    bb.mul_device(da.data_ptr(), a.size, db.data_ptr(), b.size, out.data_ptr())
    bb.device_status()
    check_product(port, a, b, out.cpu().numpy().view(np.uint64))


def mod_m61_digits(d: np.ndarray) -> int:
    """(sum d_i 2^(28 i)) mod 2^61-1 for 28-bit digits, vectorised: 2^(28 i)
    is a rotation by 28 i mod 61 bits."""
    d = d.astype(np.uint64)
    e = (np.arange(d.size, dtype=np.uint64) * np.uint64(28)) % np.uint64(61)
    low = (d & ((np.uint64(1) << (np.uint64(61) - e)) - np.uint64(1))) << e
    high = d >> (np.uint64(61) - e)
    v = (low + high) % np.uint64(M61)  # each term reduced
    while v.size > 1:  # pairwise sums, folded back below 2^61 at every level
        if v.size & 1:
            v = np.append(v, np.uint64(0))
        v = v[0::2] + v[1::2]
        v = (v & np.uint64(M61)) + (v >> np.uint64(61))
    return int(v[0]) % M61


def test_digits_beyond_the_transform(bb):
    """mul_digits above 2^31 product bits goes through u64 limbs and the block
    products."""
    rng = np.random.default_rng(SEED + 504)
    n = (1 << 30) // 28 + 1000  # two operands just over 2^30 bits each
    a, b = rand_digits(rng, n), rand_digits(rng, n)
    c = bb.mul_digits(a, b)
    assert mod_m61_digits(a) * mod_m61_digits(b) % M61 == mod_m61_digits(c)
    assert (int(a[0]) * int(b[0])) & ((1 << 28) - 1) == int(c[0])


def test_fast_pow_crosses_the_transform(bb, port):
    """A squaring chain whose last products are beyond the largest transform."""
    base, e = 3, 3 * (1 << 30) // 2  # 3^e: about 2^31.2 bits
    got = bb.fast_pow(base, e)
    assert port.mod_m61(got) == pow(base, e, M61)
    assert int(got[0]) == pow(base, e, 1 << 64)


def test_pipelined_host_api_with_a_huge_product(bb, port):
    """bgpu_mul_u64_many: a product beyond the transform between ordinary ones."""
    rng = np.random.default_rng(SEED + 505)
    pairs = [(rand_limbs(rng, 5000), rand_limbs(rng, 7000)),
             (rand_limbs(rng, BLOCK + 3), rand_limbs(rng, BLOCK + 5)),
             (rand_limbs(rng, 100), rand_limbs(rng, 60))]
    outs = bb.mul_many(pairs)
    for (a, b), c in zip(pairs, outs):
        check_product(port, a, b, c)


@pytest.fixture
def small_blocks(bb):
    bb.set_block_limbs(1 << 10)
    yield 1 << 10
    bb.set_block_limbs(0)


@pytest.mark.parametrize("na,nb", [(4096, 4096), (3000, 5000), (1025, 9000), (1 << 13, 1 << 13),
                                   (10000, 1500), (2049, 2049)])
def test_block_path_small_blocks_vs_oracle(bb, port, small_blocks, na, nb):
    """Blocks of 2^10 limbs: every product above 2^12 points runs as spectral
    sums of block products (up to four per sum at this block size, so the
    8 x 8-block case splits its longest sums) plus carry-scan accumulation;
    ragged last blocks, unbalanced block counts and squares, limb-exact
    against the oracle."""
    rng = np.random.default_rng(SEED + 300 + na + 3 * nb)
    a, b = rand_limbs(rng, na), rand_limbs(rng, nb)
    assert np.array_equal(bb.ntt_mul(a, b), port.mul(a, b))
    assert np.array_equal(bb.ntt_mul(a), port.mul(a))


def test_block_path_small_blocks_all_ones_and_device_entry(bb, port, small_blocks):
    """All-ones operands (carries across every block boundary) through the
    host API, the device entry and Digits, against the oracle."""
    torch = pytest.importorskip("torch")
    a = np.full(5000, ONES)
    b = np.full(3333, ONES)
    want = port.mul(a, b)
    assert np.array_equal(bb.ntt_mul(a, b), want)
    assert np.array_equal(bb.ntt_mul(a), port.mul(a))
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    out = torch.full((a.size + b.size,), -1, dtype=torch.int64, device="cuda")
    bb.mul_device(da.data_ptr(), a.size, db.data_ptr(), b.size, out.data_ptr(), method=bb.BGPU_METHOD_NTT)
    bb.device_status(0)
    assert np.array_equal(out.cpu().numpy().view(np.uint64), want)
    rng = np.random.default_rng(SEED + 310)
    da_, db_ = rand_digits(rng, 9000), rand_digits(rng, 7000)
    assert np.array_equal(bb.mul_digits(da_, db_), port.mul_digits(da_, db_))


def test_spectral_strict_primes_vs_one_transform(bb, port):
    """2^22-limb blocks: 2^24-point block spectra on the strict prime set
    (rows of 2^13 points), for a product and a square that also fit one
    2^26-point transform; both ways agree limb for limb."""
    rng = np.random.default_rng(SEED + 506)
    blk = 1 << 22
    a, b = rand_limbs(rng, 3 * blk + 5), rand_limbs(rng, 2 * blk + 7)
    want, want_sq = bb.ntt_mul(a, b), bb.ntt_mul(a)
    bb.set_block_limbs(blk)
    try:
        got, got_sq = bb.ntt_mul(a, b), bb.ntt_mul(a)
        got_ba = bb.ntt_mul(b, a)
    finally:
        bb.set_block_limbs(0)
    check_product(port, a, b, got)
    assert np.array_equal(got, want)
    assert np.array_equal(got_ba, want)
    assert np.array_equal(got_sq, want_sq)


def test_pairwise_block_path_vs_oracle(bb, port):
    """64-limb blocks on a 2^8-point transform split into rows of 2^4 points,
    too short for the spectral row passes: every block pair is one NTT
    product added at its offset; limb-exact against the oracle."""
    rng = np.random.default_rng(SEED + 507)
    old = bb.get_split(8)
    bb.set_block_limbs(64)
    bb.set_split(8, 4)
    try:
        a, b = rand_limbs(rng, 700), rand_limbs(rng, 300)
        got, sq = bb.ntt_mul(a, b), bb.ntt_mul(a)
    finally:
        bb.set_split(8, old)
        bb.set_block_limbs(0)
    assert np.array_equal(got, port.mul(a, b))
    assert np.array_equal(sq, port.mul(a))


def test_block_limbs_hook_rejects_bad_sizes(bb):
    for bad in (63, 100, (1 << 24) + 1, 1 << 25):
        with pytest.raises(bb.BigIntGPUError):
            bb.set_block_limbs(bad)
    bb.set_block_limbs(0)
