"""Parity of the CUDA multiply path with the oracle (bit-exact).

Every test calls through the C-ABI (bigint_b200 -> libbigint_b200.so) and
compares limb-for-limb with the oracle: the committed golden vectors made by
the reference itself, the C restatement on fresh seeded inputs, and -- at the
largest sizes where the CPU is too slow -- the residue identity
(A mod M)(B mod M) = (A*B) mod M for M = 2^61-1."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import SEED, golden_digit_cases, golden_u64_cases, rand_digits, rand_limbs
from oracle.pyoracle import digits28_to_limbs, limbs_to_int

pytestmark = pytest.mark.gpu
ONES = np.uint64(0xFFFFFFFFFFFFFFFF)
M61 = (1 << 61) - 1


def test_golden_u64_auto_and_forced(bb, golden):
    for kind, a, b, c in golden_u64_cases(golden):
        args = (a,) if b is None else (a, b)
        assert np.array_equal(bb.mul(*args), c), ("auto", kind, a.size)
        assert np.array_equal(bb.ntt_mul(*args), c), ("ntt", kind, a.size)
        if a.size + (a.size if b is None else b.size) <= 256:
            assert np.array_equal(bb.brute_mul(*args), c), ("brute", kind, a.size)


def test_golden_mul_digits(bb, golden):
    for a, b, prec, pos, c in golden_digit_cases(golden):
        for method in (bb.BGPU_METHOD_AUTO, bb.BGPU_METHOD_NTT):
            res, p = bb.mul_digits(a, a if b is None else b, prec, 7, method=method)
            assert np.array_equal(res, c) and p == pos, (a.size, prec, method)


def test_every_transform_shape(bb, port):
    """One product per supported transform length 2^5 .. 2^22 (forced NTT),
    each with uneven operand lengths so both operands have ragged tails."""
    rng = np.random.default_rng(SEED + 10)
    for log_n in range(5, 23):
        total32 = (1 << log_n) - 3  # 32-bit digits of a*b, just below N
        na = max(1, total32 // 3 // 2)
        nb = max(1, (total32 - 2 * na) // 2)
        a, b = rand_limbs(rng, na), rand_limbs(rng, nb)
        got, st = bb.ntt_mul(a, b, stats=True)
        assert st.log2_points == max(5, (2 * na + 2 * nb - 2).bit_length())
        assert np.array_equal(got, port.mul(a, b)), (log_n, na, nb)


@pytest.mark.parametrize("n", [1, 2, 7, 64, 255, 1024, 4097, 65536])
def test_all_ones_square_and_product(bb, port, n):
    ones = np.full(n, ONES)
    assert np.array_equal(bb.ntt_mul(ones), port.ntt_mul(ones))
    other = np.full(max(1, n // 3), ONES)
    assert np.array_equal(bb.ntt_mul(ones, other), port.ntt_mul(ones, other))


def test_unbalanced_pairs(bb, port):
    rng = np.random.default_rng(SEED + 11)
    for na, nb in [(16384, 256), (16384, 2048), (131072, 16384), (1, 50000), (50000, 3)]:
        a, b = rand_limbs(rng, na), rand_limbs(rng, nb)
        assert np.array_equal(bb.mul(a, b), port.mul(a, b)), (na, nb)
        assert np.array_equal(bb.mul(b, a), port.mul(b, a)), (nb, na)


def test_squares_match_products(bb, port):
    rng = np.random.default_rng(SEED + 12)
    for n in [300, 4096, 100000]:
        a = rand_limbs(rng, n)
        sq = bb.mul(a)
        assert np.array_equal(sq, bb.mul(a, a.copy()))  # distinct buffer -> general product
        assert np.array_equal(sq, port.ntt_mul(a))


def test_schoolbook_edges(bb):
    rng = np.random.default_rng(SEED + 13)
    for na, nb in [(1, 1), (1, 255), (128, 128), (100, 3)]:
        a, b = rand_limbs(rng, na), rand_limbs(rng, nb)
        want = limbs_to_int(a) * limbs_to_int(b)
        assert limbs_to_int(bb.brute_mul(a, b)) == want
        assert limbs_to_int(bb.ntt_mul(a, b)) == want


def test_zero_and_leading_zero_limbs(bb):
    z = np.zeros(5, dtype=np.uint64)
    assert bb.mul(z, np.arange(1, 9, dtype=np.uint64)).size == 0
    a = np.array([3, 0, 0, 0], dtype=np.uint64)  # leading zero limbs are ignored
    b = np.array([5, 7, 0], dtype=np.uint64)
    assert limbs_to_int(bb.mul(a, b)) == 3 * (5 + (7 << 64))


def test_output_capacity_error(bb):
    u64p = C.POINTER(C.c_uint64)
    a = np.full(600, ONES)
    out = np.zeros(10, dtype=np.uint64)
    n = C.c_size_t(0)
    rc = bb.lib.bgpu_mul_u64(a.ctypes.data_as(u64p), a.size, a.ctypes.data_as(u64p), a.size,
                             out.ctypes.data_as(u64p), out.size, C.byref(n), 0, None)
    assert rc == -5 and n.value == 1200


def test_invalid_digit_rejected(bb):
    with pytest.raises(bb.BigIntGPUError) as e:
        bb.mul_digits(np.array([1 << 28, 1], dtype=np.uint32), np.array([1], dtype=np.uint32))
    assert e.value.code == -1
    with pytest.raises(bb.BigIntGPUError):
        bb.mul_digits(np.zeros(4, np.uint32), np.array([1], dtype=np.uint32))  # all zero


def test_digits_random_vs_port(bb, port):
    rng = np.random.default_rng(SEED + 14)
    for na, nb in [(1, 1), (9, 4), (1000, 1000), (70000, 3000), (300000, 300000)]:
        a, b = rand_digits(rng, na), rand_digits(rng, nb)
        for prec in (0, 17, 2 * max(na, nb)):
            got, pos = bb.mul_digits(a, b, prec, 3)
            want, wpos = port.mul_digits(a, b, prec, 3)
            assert np.array_equal(got, want) and pos == wpos, (na, nb, prec)
        assert np.array_equal(bb.mul_digits(a), port.mul_digits(a))


def test_digits_transform_sized_by_bit_length(bb, port):
    """Digits of exactly 2^k bits (ceil(2^k / 28) digits, the top one short)
    take the same transform as 2^k-bit u64 limbs; top digits one bit longer
    take the next one.  Products exact either way."""
    rng = np.random.default_rng(SEED + 16)
    for k in (16, 20):
        nd = -(-(1 << k) // 28)
        top = (1 << k) - 28 * (nd - 1)
        a, b = rand_digits(rng, nd), rand_digits(rng, nd)
        for x in (a, b):
            x[-1] = (x[-1] & np.uint32((1 << top) - 1)) | np.uint32(1 << (top - 1))
        got, st = bb.mul_digits(a, b, method=bb.BGPU_METHOD_NTT, stats=True)
        assert st.log2_points == k - 4, (k, st.log2_points)
        assert np.array_equal(got, port.mul_digits(a, b)), k
        a[-1] |= np.uint32(1 << top)  # both 2^k + 1 bits: 2^(k-5) + 1 words each
        b[-1] |= np.uint32(1 << top)
        got, st = bb.mul_digits(a, b, method=bb.BGPU_METHOD_NTT, stats=True)
        assert st.log2_points == k - 3, (k, st.log2_points)
        assert np.array_equal(got, port.mul_digits(a, b)), k


def test_independent_products_back_to_back(bb, port):
    """BGPU_INDEPENDENT: each transform starts under the previous product's
    carry scan.  Mixed sizes, squares, a product whose operand is the previous
    output (the overlap must then be refused) and one reusing the previous
    output buffer as its own output: every product exact."""
    import torch

    rng = np.random.default_rng(SEED + 17)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    sizes = [(1 << 14, 1 << 14), (1 << 12, 1 << 15), (3000, 3000), (1 << 14, 1 << 14), (5000, 77),
             (1 << 16, 1 << 16)] * 3
    ops = [(rand_limbs(rng, na), rand_limbs(rng, nb)) for na, nb in sizes]
    dops = [(torch.from_numpy(a.view(np.int64)).to(dev), torch.from_numpy(b.view(np.int64)).to(dev))
            for a, b in ops]
    # every fourth product squares its first operand; outputs hold exactly
    # na + nb limbs, all of which the product writes
    outs = [torch.empty(2 * a.size if k % 4 == 3 else a.size + b.size, dtype=torch.int64, device=dev)
            for k, (a, b) in enumerate(ops)]
    torch.cuda.synchronize()
    flags = bb.BGPU_METHOD_AUTO | bb.BGPU_INDEPENDENT
    with torch.cuda.stream(stream):
        for k, ((a, b), (da, db)) in enumerate(zip(ops, dops)):
            sq = k % 4 == 3
            bb.mul_device(da.data_ptr(), a.size, (da if sq else db).data_ptr(), a.size if sq else b.size,
                          outs[k].data_ptr(), stream=stream.cuda_stream, method=flags)
        # chained: the operand is the previous product's output
        prev = outs[-1]
        chained = torch.empty(2 * prev.numel(), dtype=torch.int64, device=dev)
        bb.mul_device(prev.data_ptr(), prev.numel(), prev.data_ptr(), prev.numel(), chained.data_ptr(),
                      stream=stream.cuda_stream, method=flags)
    bb.device_status(stream.cuda_stream)
    for k, (a, b) in enumerate(ops):
        want = port.mul(a) if k % 4 == 3 else port.mul(a, b)
        got = outs[k].cpu().numpy().view(np.uint64)
        assert np.array_equal(got[: want.size], want) and not got[want.size:].any(), k
    p = outs[-1].cpu().numpy().view(np.uint64)
    assert port.mod_m61(p) ** 2 % M61 == port.mod_m61(chained.cpu().numpy().view(np.uint64))


def test_reference_mul_digits_regression(bb, port):
    """The reference's mul_digits regression (tests/measure_digit_bits.cpp:170-184):
    the full dispatch chain at {100, 1000, 10000, 40000} uniform 28-bit
    digits, three repetitions each, seeded like the reference."""
    rng = np.random.default_rng(SEED)
    for nd in (100, 1000, 10000, 40000):
        for _ in range(3):
            a, b = rand_digits(rng, nd), rand_digits(rng, nd)
            assert np.array_equal(bb.mul_digits(a, b), port.mul_digits(a, b)), nd


def test_headline_size_vs_port(bb, port):
    """2^24 x 2^24-bit product (the bench workload) limb-exact."""
    rng = np.random.default_rng(SEED + 15)
    a, b = rand_limbs(rng, 1 << 18), rand_limbs(rng, 1 << 18)
    got, st = bb.mul(a, b, stats=True)
    assert st.log2_points == 20
    assert np.array_equal(got, port.ntt_mul(a, b))


@pytest.mark.parametrize("bits", [1 << 26, 1 << 28])
def test_large_products_residue(bb, port, bits):
    rng = np.random.default_rng(SEED + bits.bit_length())
    n = bits // 64
    a, b = rand_limbs(rng, n), rand_limbs(rng, n)
    c = bb.mul(a, b)
    assert c.size == 2 * n
    ra, rb, rc = port.mod_m61(a), port.mod_m61(b), port.mod_m61(c)
    assert ra * rb % M61 == rc
    ones = np.full(n, ONES)
    c1 = bb.mul(ones)  # (2^k - 1)^2 = 2^2k - 2^(k+1) + 1
    k = 64 * n
    assert c1[0] == 1 and np.all(c1[1:n] == 0) and c1[n] == np.uint64(0xFFFFFFFFFFFFFFFE)
    assert np.all(c1[n + 1:] == ONES)


def test_largest_square_residue(bb, port):
    """2^30-bit square: 2^26 points, beyond the reference NTT's 2^26 x 28-bit cap."""
    rng = np.random.default_rng(SEED + 30)
    n = (1 << 30) // 64
    a = rand_limbs(rng, n)
    c = bb.mul(a)
    assert c.size == 2 * n
    ra = port.mod_m61(a)
    assert ra * ra % M61 == port.mod_m61(c)


def test_largest_general_product_residue(bb, port):
    """2^30 x 2^30-bit product (2^26 points, rows of 2^15 points through the
    one-buffer row pass): residue identity, commutativity through the other
    plane assignment, and the all-ones closed form."""
    rng = np.random.default_rng(SEED + 31)
    n = (1 << 30) // 64
    a, b = rand_limbs(rng, n), rand_limbs(rng, n)
    c, st = bb.ntt_mul(a, b, stats=True)
    assert st.log2_points == 26 and c.size == 2 * n
    assert port.mod_m61(a) * port.mod_m61(b) % M61 == port.mod_m61(c)
    assert np.array_equal(bb.ntt_mul(b, a), c)
    ones = np.full(n, ONES)
    c1 = bb.ntt_mul(ones, ones.copy())  # distinct buffers: a general product, not a square
    assert c1[0] == 1 and np.all(c1[1:n] == 0) and c1[n] == np.uint64(0xFFFFFFFFFFFFFFFE)
    assert np.all(c1[n + 1:] == ONES)


def test_device_resident_entry_point(bb, port):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(SEED + 16)
    a, b = rand_limbs(rng, 5000), rand_limbs(rng, 3000)
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    out = torch.empty(8000, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    bb.mul_device(da.data_ptr(), 5000, db.data_ptr(), 3000, out.data_ptr(), stream=s)
    bb.device_status(s)
    got = out.cpu().numpy().view(np.uint64)
    want = port.mul(a, b)
    assert np.array_equal(got[: want.size], want) and not got[want.size:].any()


def test_product_tree_matches_reference_tree(bb, golden):
    for k in range(2):
        leaves = [np.array([x], dtype=np.uint64) for x in golden[f"tree_{k:03d}_leaves"]]
        while len(leaves) > 1:
            nxt = [bb.mul(leaves[i], leaves[i + 1]) for i in range(0, len(leaves) - 1, 2)]
            if len(leaves) % 2:
                nxt.append(leaves[-1])
            leaves = nxt
        assert np.array_equal(leaves[0], digits28_to_limbs(golden[f"tree_{k:03d}_digits"]))


def test_mul_many_pipelined(bb, port):
    """bgpu_mul_u64_many: many host-resident products in one pipelined call
    (copies overlapping the multiplies), mixed sizes, squares and zeros."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(SEED + 33)
    pairs, want = [], []
    for i, (na, nb) in enumerate([(262144, 262144), (5000, 3000), (3, 2), (100, 100), (40000, 1),
                                  (262144, 262144), (70000, 65000), (1, 1)]):
        a = rand_limbs(rng, na)
        b = a if i == 3 else rand_limbs(rng, nb)
        if i == 7:
            b = np.zeros(1, dtype=np.uint64)  # a zero operand
        pairs.append((a, b))
        want.append(port.mul(a) if i == 3 else port.mul(a, b))
    outs = [torch.empty(a.size + b.size, dtype=torch.int64).pin_memory().numpy().view(np.uint64)
            for a, b in pairs]
    got = bb.mul_many(pairs, outs)
    for i, (g, w) in enumerate(zip(got, want)):
        assert np.array_equal(g, w), i
    assert all(np.array_equal(x, y) for x, y in zip(bb.mul_many(pairs), want))  # pageable buffers
