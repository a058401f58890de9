"""Batched products (bgpu_batch_plan_*): many independent products of uneven
sizes captured in one CUDA graph; each output is checked limb-exact against
the oracle, including after the graph is replayed."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED, rand_limbs

pytestmark = pytest.mark.gpu
ONES = np.uint64(0xFFFFFFFFFFFFFFFF)


def _to_dev(torch, arrs):
    return [torch.from_numpy(x.view(np.int64)).cuda() for x in arrs]


def _make_batch(torch, rng, n, lo_bits, hi_bits, ones_every=0):
    bits_a = np.exp2(rng.uniform(lo_bits, hi_bits, n)).astype(np.int64)
    bits_b = np.exp2(rng.uniform(lo_bits, hi_bits, n)).astype(np.int64)
    A, B = [], []
    for i in range(n):
        na, nb = max(1, int(bits_a[i]) // 64), max(1, int(bits_b[i]) // 64)
        if ones_every and i % ones_every == 0:
            A.append(np.full(na, ONES)), B.append(np.full(nb, ONES))
        else:
            A.append(rand_limbs(rng, na)), B.append(rand_limbs(rng, nb))
    return A, B


def test_batch_plan_uneven_sizes_and_replay(bb, port):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(SEED + 40)
    A, B = _make_batch(torch, rng, 300, 10, 19, ones_every=17)
    A[5] = A[4]  # include squares: same buffer passed twice
    dA, dB = _to_dev(torch, A), _to_dev(torch, B)
    dB[5] = dA[5]
    outs = [torch.full((a.size + (a.size if i == 5 else b.size),), -1, dtype=torch.int64, device="cuda")
            for i, (a, b) in enumerate(zip(A, B))]
    prods = []
    for i in range(len(A)):
        nb = A[i].size if i == 5 else B[i].size
        prods.append((dA[i].data_ptr(), A[i].size, dB[i].data_ptr(), nb, outs[i].data_ptr()))
    plan = bb.BatchPlan(prods)
    assert plan.launches >= 2
    s = torch.cuda.Stream()
    for rep in range(2):
        for o in outs:
            o.fill_(-1)
        plan.run(s.cuda_stream)
        bb.device_status(s.cuda_stream)
        for i in range(len(A)):
            got = outs[i].cpu().numpy().view(np.uint64)
            want = port.mul(A[i]) if i == 5 else port.mul(A[i], B[i])
            assert np.array_equal(got[: want.size], want) and not got[want.size:].any(), (rep, i)
    plan.close()


def test_mul_batch_device_one_shot(bb, port):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(SEED + 41)
    A, B = _make_batch(torch, rng, 64, 6, 15)
    dA, dB = _to_dev(torch, A), _to_dev(torch, B)
    outs = [torch.empty(a.size + b.size, dtype=torch.int64, device="cuda") for a, b in zip(A, B)]
    bb.mul_batch_device([(dA[i].data_ptr(), A[i].size, dB[i].data_ptr(), B[i].size, outs[i].data_ptr())
                         for i in range(len(A))])
    for i in range(len(A)):
        got = outs[i].cpu().numpy().view(np.uint64)
        want = port.mul(A[i], B[i])
        assert np.array_equal(got[: want.size], want), i


def test_batch_rejects_bad_descriptor(bb):
    with pytest.raises(bb.BigIntGPUError) as e:
        bb.BatchPlan([(0, 4, 0, 4, 0)])
    assert e.value.code == -1


def _run_plan_and_check(bb, port, torch, A, B, square_idx=(), flags=0):
    dA, dB = _to_dev(torch, A), _to_dev(torch, B)
    for i in square_idx:
        dB[i] = dA[i]
    outs = [torch.full((a.size + (a.size if i in square_idx else b.size),), -1, dtype=torch.int64,
                       device="cuda") for i, (a, b) in enumerate(zip(A, B))]
    prods = [(dA[i].data_ptr(), A[i].size, dB[i].data_ptr(), A[i].size if i in square_idx else B[i].size,
              outs[i].data_ptr()) for i in range(len(A))]
    plan = bb.BatchPlan(prods, flags=flags)
    launches = plan.launches
    for _ in range(2):
        plan.run(0)
        bb.device_status(0)
    plan.close()
    for i in range(len(A)):
        got = outs[i].cpu().numpy().view(np.uint64)
        want = port.mul(A[i]) if i in square_idx else port.mul(A[i], B[i])
        assert np.array_equal(got[: want.size], want) and not got[want.size:].any(), i
    return launches


def test_batch_one_launch_per_pass_with_small_products(bb, port):
    """Every length qualifies for the mixed-length launches: four kernels in
    all, the schoolbook and Karatsuba products riding in the row and inverse
    passes, squares among them; run twice (state reset between runs)."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(SEED + 42)
    A, B = _make_batch(torch, rng, 200, 6, 17, ones_every=13)
    A[3] = A[2]
    assert _run_plan_and_check(bb, port, torch, A, B, square_idx=(3,)) == 4


def test_batch_per_class_flag(bb, port):
    """BGPU_BATCH_PER_CLASS: the same kind of batch as the mixed-launch test,
    every class on its own four launches (graph branches), same results."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(SEED + 42)
    A, B = _make_batch(torch, rng, 200, 6, 17, ones_every=13)
    A[3] = A[2]
    launches = _run_plan_and_check(bb, port, torch, A, B, square_idx=(3,), flags=bb.BGPU_BATCH_PER_CLASS)
    assert launches > 4


def test_batch_with_a_long_class_runs_per_class(bb, port):
    """A transform too long for the mixed-length launches (2^20 points) sends
    the batch back to one set of launches per class on graph branches."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(SEED + 43)
    A, B = _make_batch(torch, rng, 40, 8, 14)
    A.append(rand_limbs(rng, 1 << 18))
    B.append(rand_limbs(rng, 1 << 18))
    assert _run_plan_and_check(bb, port, torch, A, B) > 4


def test_batch_of_small_products_only(bb, port):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(SEED + 44)
    A, B = _make_batch(torch, rng, 100, 6, 13)
    _run_plan_and_check(bb, port, torch, A, B)


def test_batch_more_products_than_one_class_launch_slice(bb, port):
    """20000 products of several lengths in the mixed launches (the per-class
    launches slice classes above 16384 products; the mixed ones take every
    CTA in one grid); a sample checked against the oracle, every product by
    its residue."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(SEED + 45)
    n = 20000
    na = rng.integers(1, 1500, n)  # schoolbook, Karatsuba and four transform lengths
    nb = rng.integers(1, 1500, n)
    big = rng.integers(0, 2**64, int(na.sum() + nb.sum()), dtype=np.uint64, endpoint=False)
    offs_a = np.concatenate([[0], np.cumsum(na)[:-1]])
    offs_b = np.concatenate([[0], np.cumsum(nb)[:-1]]) + na.sum()
    outn = na + nb
    offs_o = np.concatenate([[0], np.cumsum(outn)[:-1]])
    dbig = torch.from_numpy(big.view(np.int64)).cuda()
    dout = torch.full((int(outn.sum()),), -1, dtype=torch.int64, device="cuda")
    bi, bo = dbig.data_ptr(), dout.data_ptr()
    plan = bb.BatchPlan([(bi + 8 * int(offs_a[i]), int(na[i]), bi + 8 * int(offs_b[i]), int(nb[i]),
                          bo + 8 * int(offs_o[i])) for i in range(n)])
    assert plan.launches == 4
    plan.run(0)
    bb.device_status(0)
    plan.close()
    host = dout.cpu().numpy().view(np.uint64)
    M = (1 << 61) - 1
    for i in range(n):
        a = big[offs_a[i]:offs_a[i] + na[i]]
        b = big[offs_b[i]:offs_b[i] + nb[i]]
        c = host[offs_o[i]:offs_o[i] + outn[i]]
        assert port.mod_m61(a) * port.mod_m61(b) % M == port.mod_m61(c), i
        if i % 997 == 0:
            assert np.array_equal(np.trim_zeros(c, "b"), port.mul(a, b)), i
