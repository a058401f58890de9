"""Generate the golden vectors in this folder by running the UNMODIFIED
reference multiply path (oracle/_ref/libbigint_ref.so, built from the
reference sources by oracle/build.py).

The reference ships no golden vectors or known-answer files; its own test
(tests/measure_digit_bits.cpp) cross-checks fft::mul against ntt::mul on
seeded random and all-ones inputs (seed 0x9e3779b97f4a7c15, :140; all-ones
operands, :65-85).  These fixtures record the reference's own outputs for the
same kinds of inputs (seeded with that seed value through numpy's PCG64), so
the oracle and the GPU path can be pinned on machines without the reference.

Run from the repo root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.pyoracle import Reference  # noqa: E402

SEED = 0x9E3779B97F4A7C15
ALL = np.uint64(0xFFFFFFFFFFFFFFFF)


def rand_limbs(rng, n, top=True):
    x = rng.integers(0, 2**64, n, dtype=np.uint64, endpoint=False)
    if top:
        x[-1] |= np.uint64(1 << 63)
    return x


def rand_digits(rng, n):
    d = rng.integers(0, 1 << 28, n, dtype=np.uint32)
    if d[-1] == 0:
        d[-1] = 1
    return d


def main() -> None:
    ref = Reference()
    ref.init_thread_pool(8)
    rng = np.random.default_rng(SEED)
    arrays: dict[str, np.ndarray] = {}

    # u64-limb products through the dispatcher (_mul) and through ntt::mul.
    shapes = [(1, 1), (2, 1), (3, 3), (16, 16), (64, 100), (128, 128), (129, 127), (300, 300),
              (1000, 1000), (2048, 512), (4096, 4096), (5000, 77)]
    cases = []
    for na, nb in shapes:
        cases.append(("rand", rand_limbs(rng, na), rand_limbs(rng, nb)))
    for na, nb in [(1, 1), (100, 100), (4096, 4096), (3000, 17)]:
        cases.append(("ones", np.full(na, ALL), np.full(nb, ALL)))
    for n in [777, 4096]:
        a = rand_limbs(rng, n)
        cases.append(("square", a, a))
    cases.append(("ones_square", np.full(2048, ALL), None))
    # structured values: powers of two, sparse limbs, a single top bit
    pw = np.zeros(513, dtype=np.uint64)
    pw[-1] = np.uint64(1)
    cases.append(("pow2", pw, rand_limbs(rng, 700)))
    sp = rand_limbs(rng, 1500)
    sp[100:1400] = 0
    cases.append(("sparse", sp, rand_limbs(rng, 1100)))
    cases.append(("one", np.array([1], dtype=np.uint64), rand_limbs(rng, 2000)))

    for i, (kind, a, b) in enumerate(cases):
        if b is None or kind == "square":
            c_mul = ref.mul(a)
            c_ntt = ref.ntt_mul(a)
            arrays[f"u64_{i:03d}_b"] = np.zeros(0, dtype=np.uint64)
        else:
            c_mul = ref.mul(a, b)
            c_ntt = ref.ntt_mul(a, b)
            arrays[f"u64_{i:03d}_b"] = b
        assert np.array_equal(c_mul, c_ntt), (kind, a.size)
        arrays[f"u64_{i:03d}_a"] = a
        arrays[f"u64_{i:03d}_c"] = c_mul
        arrays[f"u64_{i:03d}_kind"] = np.array(kind)

    # mul_digits with output_precision / point_pos (mul.h:223-318).
    j = 0
    for na, nb in [(5, 3), (100, 100), (1000, 400), (3000, 2000)]:
        da, db = rand_digits(rng, na), rand_digits(rng, nb)
        da[: min(3, na - 1)] = 0  # low zero digits exercise tail_zero handling
        for prec in [0, 1, 10, 500, 2500]:
            for square in (False, True):
                if square:
                    res, pos = ref.mul_digits(da, None, prec, 7)
                else:
                    res, pos = ref.mul_digits(da, db, prec, 7)
                arrays[f"dig_{j:03d}_a"] = da
                arrays[f"dig_{j:03d}_b"] = np.zeros(0, np.uint32) if square else db
                arrays[f"dig_{j:03d}_prec"] = np.array(prec)
                arrays[f"dig_{j:03d}_pos"] = np.array(pos)
                arrays[f"dig_{j:03d}_c"] = res
                j += 1

    # BigInt pairwise product tree (the binary-splitting caller pattern).
    for k, n in enumerate([64, 1000]):
        leaves = rng.integers(1 << 32, 2**64, n, dtype=np.uint64, endpoint=False)
        arrays[f"tree_{k:03d}_leaves"] = leaves
        arrays[f"tree_{k:03d}_digits"] = ref.product_tree_digits(leaves)

    out = os.path.join(HERE, "golden.npz")
    np.savez_compressed(out, **arrays)
    print(f"wrote {out}: {len(cases)} u64 cases, {j} mul_digits cases, 2 trees, "
          f"{os.path.getsize(out) / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
