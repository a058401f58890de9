"""CPU model of the spectral block products beyond the largest transform
(huge_spectral in bigint_b200/csrc/engine.cu; k_chunks_merge and the carry
scan's chunk format in bigint_b200/csrc/ntt_kernels.cu), in Python integers.

Both operands are cut into blocks of S limbs; output block k is
C_k = sum_{i+j=k} A_i B_j, formed as sums of at most `tmax` block products
(a square's off-diagonal pairs once, doubled), each carried into the result's
window of 2S + 1 limbs at limb kS together with what the window holds.  The
model checks, for random and all-ones operands, unbalanced block counts and
squares: that no sum's carry leaves its window (the reason the carry scan
covers the window alone), that the first sum of each C_k finds nothing above
the window's first S + 1 limbs (the reason its merge reads only those), and
that the result is the product.  A second model runs the merge on the chunk
format itself: 8 coefficients of up to 91 bits per chunk as 4 limbs plus a
spill, doubled and added to the window limbs, then carried; and the CRT
bound that sets tmax."""
from __future__ import annotations

import random

import pytest

LIMB = 64
P_LAZY = (469762049, 754974721, 998244353)
P_STRICT = (469762049, 1811939329, 2013265921)
MAX_TERMS = 4  # kMaxSpecTerms


def spectral_terms(primes, s_limbs: int) -> int:
    """engine.cu spectral_terms: block products per sum under the CRT bound."""
    m = primes[0] * primes[1] * primes[2]
    per = (2**32 - 1) ** 2 * (2 * s_limbs)
    return min((m - 1) // per, MAX_TERMS)


def test_terms_per_sum():
    assert spectral_terms(P_STRICT, 1 << 24) == 2   # the default 2^30-bit blocks
    assert spectral_terms(P_STRICT, 1 << 22) == 4   # the strict-prime test blocks
    assert spectral_terms(P_LAZY, 1 << 10) == 4     # the small test blocks
    # the bound itself: two full block products' coefficients fit, three do not
    m = P_STRICT[0] * P_STRICT[1] * P_STRICT[2]
    assert 2 * (2 << 24) * (2**32 - 1) ** 2 < m < 3 * (2 << 24) * (2**32 - 1) ** 2


def blocks(x: int, nlimbs: int, s: int) -> list[int]:
    n = -(-nlimbs // s)
    return [(x >> (LIMB * s * i)) & ((1 << (LIMB * s)) - 1) for i in range(n)]


def spectral_product(a: int, na: int, b: int, nb: int, s: int, tmax: int, square: bool) -> int:
    L = na + nb
    A = blocks(a, na, s)
    B = A if square else blocks(b, nb, s)
    out = 0
    for k in range(len(A) + len(B) - 1):
        once, twice = [], []
        for i in range(max(0, k - (len(B) - 1)), min(k, len(A) - 1) + 1):
            j = k - i
            if not square:
                once.append((i, j))
            elif i < j:
                twice.append((i, j))
            elif i == j:
                once.append((i, j))
        off = k * s
        win = min(2 * s + 1, L - off)
        first = True
        for pairs, doubled in ((once, False), (twice, True)):
            for g in range(0, len(pairs), tmax):
                c = sum(A[i] * B[j] for i, j in pairs[g:g + tmax])
                if doubled:
                    c *= 2
                window = (out >> (LIMB * off)) & ((1 << (LIMB * win)) - 1)
                assert out >> (LIMB * (off + win)) == 0  # nothing above the window yet
                if first:
                    keep = 0 if k == 0 else min(s + 1, win)
                    assert window >> (LIMB * keep) == 0  # the first merge reads `keep` limbs
                    first = False
                new = window + c
                assert new < 1 << (LIMB * win)  # no carry leaves the window
                out += (new - window) << (LIMB * off)
    return out


def rand_int(rng: random.Random, nlimbs: int) -> int:
    return rng.getrandbits(LIMB * nlimbs) | (1 << (LIMB * nlimbs - 1))


@pytest.mark.parametrize("na,nb,s,tmax", [(16, 16, 4, 2), (13, 5, 4, 2), (5, 13, 4, 2), (33, 33, 4, 2),
                                          (40, 9, 8, 1), (24, 24, 3, 4), (7, 7, 8, 2), (64, 64, 4, 3)])
def test_spectral_blocks_make_the_product(na, nb, s, tmax):
    rng = random.Random(na * 1000 + nb * 10 + s)
    a, b = rand_int(rng, na), rand_int(rng, nb)
    assert spectral_product(a, na, b, nb, s, tmax, False) == a * b
    assert spectral_product(a, na, a, na, s, tmax, True) == a * a


@pytest.mark.parametrize("n,s,tmax", [(16, 4, 2), (17, 4, 2), (31, 8, 2), (40, 4, 4)])
def test_all_ones_fill_every_window(n, s, tmax):
    """(2^k - 1)^2 and (2^k - 1)(2^m - 1): the largest block products, with
    carry runs through every window."""
    a = (1 << (LIMB * n)) - 1
    b = (1 << (LIMB * (n // 2 + 1))) - 1
    assert spectral_product(a, n, a, n, s, tmax, True) == a * a
    assert spectral_product(a, n, b, n // 2 + 1, s, tmax, False) == a * b


def chunk_format(coefs: list[int]):
    """The inverse pass's chunk sums: 8 coefficients (digit positions 32 i)
    per chunk as 4 limbs and a spill (bits above 256)."""
    chunks = []
    for c0 in range(0, len(coefs), 8):
        v = sum(x << (32 * i) for i, x in enumerate(coefs[c0:c0 + 8]))
        chunks.append(([(v >> (64 * t)) & (2**64 - 1) for t in range(4)], v >> 256))
    return chunks


def merge(chunks, add: list[int], twice: bool):
    """k_chunks_merge on one product's chunks (u64 arithmetic, as the kernel)."""
    M = 2**64 - 1
    out = []
    n = len(chunks)
    for c, (s, sp) in enumerate(chunks):
        s = list(s)
        if twice:
            sp = ((sp << 1) | (s[3] >> 63)) & M
            s = [((s[t] << 1) | (s[t - 1] >> 63 if t else 0)) & M for t in range(4)]
        cy = 0
        for t in range(4):
            w = add[4 * c + t] if 4 * c + t < len(add) else 0
            u = s[t] + w
            r = u + cy
            cy = (u > M) | (r > M)  # the kernel's (t < w) | (r < t) on wrapped values
            s[t] = r & M
        sp += cy
        if c == n - 1 and len(add) > 4 * c + 4:
            sp += add[4 * c + 4]
        assert sp < 1 << 61
        out.append((s, sp))
    return out


def carried_value(chunks) -> int:
    """What the carry scan computes: chunk c contributes its limbs at 256 c
    bits and its spill at 256 (c + 1)."""
    v = 0
    for c, (s, sp) in enumerate(chunks):
        v += sum(x << (64 * t) for t, x in enumerate(s)) << (256 * c)
        v += sp << (256 * (c + 1))
    return v


@pytest.mark.parametrize("twice", [False, True])
def test_merge_on_chunk_format(twice):
    rng = random.Random(5 + twice)
    m = P_STRICT[0] * P_STRICT[1] * P_STRICT[2]
    for trial in range(20):
        n = 8 * rng.randint(1, 6)
        coefs = [rng.randrange(m) if trial % 3 else m - 1 for _ in range(n)]  # up to the CRT range
        chunks = chunk_format(coefs)
        value = sum(x << (32 * i) for i, x in enumerate(coefs))
        # window limbs: any value over the chunks' n / 2 limbs; the one past
        # them (the window's top limb) is 0 before the window's first sum and
        # after it below the number of block products already carried there
        add = [rng.getrandbits(64) for _ in range(rng.randint(0, n // 2))]
        if rng.random() < 0.5:
            add = [rng.getrandbits(64) for _ in range(n // 2)] + [rng.randrange(MAX_TERMS + 1)]
        addv = sum(x << (64 * i) for i, x in enumerate(add))
        merged = merge(chunks, add, twice)
        assert carried_value(merged) == (2 if twice else 1) * value + addv
