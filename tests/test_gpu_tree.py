"""Product tree (the binary-splitting caller pattern, examples/pi.cpp:41-80)
on the GPU: checked against the reference's own BigInt tree (golden vectors),
the oracle's tree, and at 2^20 leaves by the residue identity."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED
from oracle.pyoracle import digits28_to_limbs

pytestmark = pytest.mark.gpu
M61 = (1 << 61) - 1


def test_tree_matches_reference_bigint_tree(bb, golden):
    for k in range(2):
        leaves = golden[f"tree_{k:03d}_leaves"]
        assert np.array_equal(bb.product_tree(leaves), digits28_to_limbs(golden[f"tree_{k:03d}_digits"]))


@pytest.mark.parametrize("n", [1, 2, 3, 7, 1000, 4097, 1 << 16])
def test_tree_matches_oracle(bb, port, n):
    rng = np.random.default_rng(SEED + n)
    leaves = rng.integers(1 << 32, 2**64, n, dtype=np.uint64, endpoint=False)
    assert np.array_equal(bb.product_tree(leaves), port.product_tree(leaves))


def test_tree_full_size_residue(bb, port):
    """2^20 leaves in [2^32, 2^64) -> a ~2^26-bit product (the tree workload)."""
    rng = np.random.default_rng(SEED + 5)
    leaves = rng.integers(1 << 32, 2**64, 1 << 20, dtype=np.uint64, endpoint=False)
    got = bb.product_tree(leaves)
    r = 1
    for x in leaves.tolist():
        r = r * (x % M61) % M61
    assert port.mod_m61(got) == r
    assert got.size > (1 << 19)


def test_tree_all_ones_leaves(bb, port):
    leaves = np.full(3000, np.uint64(0xFFFFFFFFFFFFFFFF))
    assert np.array_equal(bb.product_tree(leaves), port.product_tree(leaves))
