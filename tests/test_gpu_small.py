"""Small-product kernels (schoolbook and Karatsuba, one CTA per product):
single products through the C-ABI, batch plans and product-tree levels that
use them, each checked limb-exact against the oracle.  All-ones operands make
every column sum maximal and every carry run the full length."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED, rand_digits, rand_limbs

pytestmark = pytest.mark.gpu
ONES = np.uint64(0xFFFFFFFFFFFFFFFF)

SIZES = [(1, 1), (1, 2), (2, 1), (3, 5), (17, 16), (31, 97), (100, 100), (127, 129),
         (128, 128), (1, 256), (256, 1), (200, 37), (255, 256), (256, 256)]


@pytest.fixture
def tuned(bb):
    """Restore the crossovers a test changes."""
    keys = (bb.BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS, bb.BGPU_TUNE_BATCH_SCHOOLBOOK_MAX_LIMBS,
            bb.BGPU_TUNE_KARATSUBA_MAX_LIMBS, bb.BGPU_TUNE_BATCH_KARATSUBA_MAX_LIMBS)
    saved = {k: bb.get_tuning(k) for k in keys}
    yield bb
    for k, v in saved.items():
        bb.set_tuning(k, v)


@pytest.mark.parametrize("na,nb", SIZES)
def test_karatsuba_single(bb, port, na, nb):
    rng = np.random.default_rng(SEED + 60 + na * 1000 + nb)
    a, b = rand_limbs(rng, na), rand_limbs(rng, nb)
    got, st = bb.karatsuba_mul(a, b, stats=True)
    assert st.method == bb.BGPU_METHOD_KARATSUBA
    assert np.array_equal(got, port.mul(a, b))
    assert np.array_equal(bb.karatsuba_mul(a), port.mul(a))  # square
    oa, ob = np.full(na, ONES), np.full(nb, ONES)
    assert np.array_equal(bb.karatsuba_mul(oa, ob), port.mul(oa, ob))


@pytest.mark.parametrize("na,nb", [(1, 1), (1, 255), (128, 128), (100, 3), (200, 56), (64, 64)])
def test_schoolbook_carry_chains(bb, port, na, nb):
    """All-ones and 2^(64n) - 2^(64k) operands: carries that ripple across the
    whole product through the block-wide carry resolution."""
    oa, ob = np.full(na, ONES), np.full(nb, ONES)
    assert np.array_equal(bb.brute_mul(oa, ob), port.mul(oa, ob))
    a = np.full(na, ONES)
    a[: na // 2] = 0
    assert np.array_equal(bb.brute_mul(a, ob), port.mul(a, ob))
    # (2^64 - 1) * (2^(64 nb) - 1): one generate, then a full propagate run
    assert np.array_equal(bb.brute_mul(np.array([ONES]), ob), port.mul(np.array([ONES]), ob))


def test_karatsuba_rejects_oversize(bb):
    with pytest.raises(bb.BigIntGPUError):
        bb.karatsuba_mul(np.ones(257, dtype=np.uint64), np.ones(3, dtype=np.uint64))


def test_auto_uses_tuned_crossovers(tuned, port):
    bb = tuned
    rng = np.random.default_rng(SEED + 61)
    bb.set_tuning(bb.BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS, 64)
    bb.set_tuning(bb.BGPU_TUNE_KARATSUBA_MAX_LIMBS, 512)
    for (na, nb), want in [((20, 30), bb.BGPU_METHOD_SCHOOLBOOK), ((200, 250), bb.BGPU_METHOD_KARATSUBA), ((200, 300), bb.BGPU_METHOD_NTT),
                           ((256, 256), bb.BGPU_METHOD_KARATSUBA), ((300, 100), bb.BGPU_METHOD_NTT)]:
        a, b = rand_limbs(rng, na), rand_limbs(rng, nb)
        got, st = bb.mul(a, b, stats=True)
        assert st.method == want, (na, nb)
        assert np.array_equal(got, port.mul(a, b))


def test_mul_digits_small_methods(bb, port):
    rng = np.random.default_rng(SEED + 62)
    for nd in (1, 9, 500, 580):
        a, b = rand_digits(rng, nd), rand_digits(rng, nd // 2 + 1)
        want = port.mul_digits(a, b)
        for m in (bb.BGPU_METHOD_SCHOOLBOOK, bb.BGPU_METHOD_KARATSUBA):
            la, lb = (nd * 28 + 63) // 64, ((nd // 2 + 1) * 28 + 63) // 64
            if m == bb.BGPU_METHOD_SCHOOLBOOK and la + lb > 256:
                continue
            got = bb.mul_digits(a, b, method=m)
            assert np.array_equal(got, want), (nd, m)


def test_batch_with_karatsuba_class(tuned, port):
    torch = pytest.importorskip("torch")
    bb = tuned
    bb.set_tuning(bb.BGPU_TUNE_BATCH_SCHOOLBOOK_MAX_LIMBS, 96)
    bb.set_tuning(bb.BGPU_TUNE_BATCH_KARATSUBA_MAX_LIMBS, 512)
    rng = np.random.default_rng(SEED + 63)
    sizes = [(int(rng.integers(1, 257)), int(rng.integers(1, 257))) for _ in range(200)]
    sizes += [(256, 256), (1, 1), (300, 20), (40, 40)]
    A = [rand_limbs(rng, na) for na, _ in sizes]
    B = [np.full(nb, ONES) if i % 7 == 0 else rand_limbs(rng, nb) for i, (_, nb) in enumerate(sizes)]
    dA = [torch.from_numpy(x.view(np.int64)).cuda() for x in A]
    dB = [torch.from_numpy(x.view(np.int64)).cuda() for x in B]
    outs = [torch.full((a.size + b.size,), -1, dtype=torch.int64, device="cuda") for a, b in zip(A, B)]
    prods = [(dA[i].data_ptr(), A[i].size, dB[i].data_ptr(), B[i].size, outs[i].data_ptr())
             for i in range(len(A))]
    plan = bb.BatchPlan(prods)
    s = torch.cuda.Stream()
    plan.run(s.cuda_stream)
    bb.device_status(s.cuda_stream)
    for i in range(len(A)):
        got = outs[i].cpu().numpy().view(np.uint64)
        want = port.mul(A[i], B[i])
        assert np.array_equal(got[: want.size], want) and not got[want.size:].any(), (i, sizes[i])
    plan.close()


@pytest.mark.parametrize("n", [5000, 1 << 14])
def test_tree_with_karatsuba_levels(tuned, port, n):
    bb = tuned
    bb.set_tuning(bb.BGPU_TUNE_BATCH_SCHOOLBOOK_MAX_LIMBS, 32)
    bb.set_tuning(bb.BGPU_TUNE_BATCH_KARATSUBA_MAX_LIMBS, 512)
    rng = np.random.default_rng(SEED + 64 + n)
    leaves = rng.integers(1 << 32, 2**64, n, dtype=np.uint64, endpoint=False)
    assert np.array_equal(bb.product_tree(leaves), port.product_tree(leaves))
    ones = np.full(n // 4, ONES)
    assert np.array_equal(bb.product_tree(ones), port.product_tree(ones))
