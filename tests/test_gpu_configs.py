"""The benchmark configurations at their stated sizes, limb-exact against the
reference's own CPU code (oracle/_ref, the unmodified reference sources):

* the batched uneven workload: all 4096 products of operands log-uniform in
  [2^10, 2^22] bits, one batch plan, against `bigint::mul::_mul`
  (include/bigint/mul.h:208-220) -- the reference runs in a pool of worker
  processes, each rebuilding its products from their seeds;
* the product tree: 2^20 leaves in [2^32, 2^64), against the reference's
  pairwise `BigInt::operator*` tree (examples/pi.cpp:41-80 is the pattern);
* the size sweep's largest products the reference's NTT can do: 2^26- and
  2^28-bit squares and general products, uniform and all-ones limbs, and the
  2^24 x 2^21 unbalanced pair, against `ntt::mul`
  (src/mul/ntt_multithread.cpp:444-530)."""
from __future__ import annotations

import hashlib
import multiprocessing as mp
import os

import numpy as np
import pytest

from conftest import SEED

pytestmark = pytest.mark.gpu
ONES = np.uint64(0xFFFFFFFFFFFFFFFF)


def _digest(x) -> str:
    return hashlib.sha1(np.trim_zeros(np.ascontiguousarray(x, dtype=np.uint64), "b").tobytes()).hexdigest()


def _reference_batch_digests(job):
    """Worker (a spawned process): the reference's _mul of the batched
    products `idx`, rebuilt from their seeds; returns {index: digest}."""
    idx, threads = job
    import bench
    from oracle.pyoracle import Reference

    ref = Reference()
    ref.init_thread_pool(threads)
    na, nb = bench.batched_sizes()
    out = {}
    for i in idx:
        a, b = bench.batched_operands(i, na[i], nb[i])
        out[i] = _digest(ref.mul(a, b))
    return out


def test_batched_4096_uneven_products_vs_reference(bb, reference):
    torch = pytest.importorskip("torch")
    import bench

    big, offs_a, na, offs_b, nb = bench.batched_inputs()
    nprod = na.size
    # the reference first, in spawned workers (no process forks after CUDA starts)
    cores = bench.physical_cores()
    workers = max(1, min(16, cores // 2))
    order = np.argsort(-(na + nb))  # largest first, dealt round-robin
    jobs = [([int(i) for i in order[w::workers]], 2) for w in range(workers)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        want = {}
        for part in pool.map(_reference_batch_digests, jobs):
            want.update(part)
    dbig = torch.from_numpy(big.view(np.int64)).cuda()
    outn = na + nb
    offs_o = np.concatenate([[0], np.cumsum(outn)[:-1]])
    dout = torch.full((int(outn.sum()),), -1, dtype=torch.int64, device="cuda")
    bi, bo = dbig.data_ptr(), dout.data_ptr()
    prods = [(bi + 8 * int(offs_a[i]), int(na[i]), bi + 8 * int(offs_b[i]), int(nb[i]), bo + 8 * int(offs_o[i]))
             for i in range(nprod)]
    plan = bb.BatchPlan(prods)
    try:
        plan.run(0)
        bb.device_status(0)
    finally:
        plan.close()
    host = dout.cpu().numpy().view(np.uint64)
    bad = [i for i in range(nprod) if _digest(host[offs_o[i]:offs_o[i] + outn[i]]) != want[i]]
    assert not bad, f"{len(bad)} of {nprod} batched products differ from the reference, first {bad[:5]}"


def test_product_tree_2p20_leaves_vs_reference(bb, reference):
    import bench

    rng = np.random.default_rng(SEED + 5)
    leaves = rng.integers(1 << 32, 2**64, 1 << 20, dtype=np.uint64, endpoint=False)
    got = bb.product_tree(leaves)
    want = reference.product_tree_digits(leaves)
    assert np.array_equal(bench.limbs_to_digits28_np(got), want)


@pytest.mark.parametrize("abits,bbits", [(1 << 26, 1 << 26), (1 << 28, 1 << 28), (1 << 24, 1 << 21)])
@pytest.mark.parametrize("fill", ["uniform", "all-ones"])
def test_sweep_large_products_vs_reference_ntt(bb, reference, abits, bbits, fill):
    rng = np.random.default_rng(SEED + 2 + abits.bit_length() + bbits.bit_length())
    na, nb = abits // 64, bbits // 64
    if fill == "uniform":
        a = rng.integers(0, 2**64, na, dtype=np.uint64, endpoint=False)
        b = rng.integers(0, 2**64, nb, dtype=np.uint64, endpoint=False)
        a[-1] |= np.uint64(1 << 63)
        b[-1] |= np.uint64(1 << 63)
    else:
        a, b = np.full(na, ONES), np.full(nb, ONES)
    assert np.array_equal(bb.ntt_mul(a, b), reference.ntt_mul(a, b))
    if abits == bbits:
        assert np.array_equal(bb.ntt_mul(a), reference.ntt_mul(a))
