"""Host <-> device copies of the host API.

Pageable operands above 256 KiB go through the engine's ring of four 4 MiB
page-locked slots (host copies split over a thread pool); page-locked ones go
straight to the copy engines.  Both routes must give the same products, the
28-bit check of Digits must see every digit on either route, and a rejected
call must leave the ring usable."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED, rand_digits, rand_limbs

pytestmark = pytest.mark.gpu
M61 = (1 << 61) - 1
SLOT_LIMBS = (4 << 20) // 8
DIRECT_LIMBS = (256 << 10) // 8
_pinned = []  # page-locked storage behind the views handed out below


def pinned_like(x: np.ndarray) -> np.ndarray:
    import torch

    t = torch.empty(x.nbytes, dtype=torch.uint8).pin_memory()
    _pinned.append(t)
    p = t.numpy().view(x.dtype)
    p[:] = x
    return p


@pytest.fixture(autouse=True)
def _release_pinned():
    yield
    _pinned.clear()


@pytest.mark.parametrize("n", [DIRECT_LIMBS - 1, DIRECT_LIMBS + 1, SLOT_LIMBS + 1,
                               3 * SLOT_LIMBS + 5, 5 * SLOT_LIMBS - 3])
def test_pageable_and_page_locked_agree(bb, port, n):
    """Sizes either side of the direct-copy limit and of the slot size, and
    more chunks than slots (the ring wraps on input and output)."""
    rng = np.random.default_rng(SEED + 200 + n % 97)
    a, b = rand_limbs(rng, n), rand_limbs(rng, n // 2 + 1)
    c = bb.mul(a, b)
    assert port.mod_m61(a) * port.mod_m61(b) % M61 == port.mod_m61(c)
    pa, pb = pinned_like(a), pinned_like(b)
    out = pinned_like(np.zeros(a.size + b.size, np.uint64))
    assert np.array_equal(bb.mul(pa, pb, out=out), c)
    assert np.array_equal(bb.mul(a, pb), c)  # one operand of each kind
    sq = bb.mul(a)
    assert np.array_equal(bb.mul(pa), sq)


@pytest.mark.parametrize("pos", [0, 65535, 65536, (1 << 20) - 1, 1 << 20, 3 * (1 << 20) + 7, -1])
def test_bad_digit_seen_anywhere(bb, pos):
    """A digit >= 2^28 at a piece boundary (64 Ki digits), at a slot
    boundary (1 Mi digits), in a later slot and at the top is rejected on both
    routes, and the next valid call still multiplies correctly."""
    rng = np.random.default_rng(SEED + 300)
    n = 3 * (1 << 20) + 11
    a, b = rand_digits(rng, n), rand_digits(rng, 1000)
    a[pos] |= np.uint32(1 << 28)
    for x in (a, pinned_like(a)):
        with pytest.raises(bb.BigIntGPUError) as e:
            bb.mul_digits(x, b)
        assert e.value.code == -1
        with pytest.raises(bb.BigIntGPUError):
            bb.mul_digits(b, x)
    a[pos] &= np.uint32((1 << 28) - 1)
    if a[-1] == 0:
        a[-1] = 1
    good = bb.mul_digits(a, b)
    assert np.array_equal(bb.mul_digits(pinned_like(a), pinned_like(b)), good)
    assert np.array_equal(bb.mul_digits(b, a), good)


def test_digits_staged_vs_port(bb, port):
    """A Digits product spanning several slots on input and output, exact."""
    rng = np.random.default_rng(SEED + 301)
    a, b = rand_digits(rng, (5 << 20) // 4 + 3), rand_digits(rng, 70001)
    assert np.array_equal(bb.mul_digits(a, b), port.mul_digits(a, b))


def test_many_calls_reuse_ring(bb, port):
    """Alternating sizes and routes over one ring: every product exact."""
    rng = np.random.default_rng(SEED + 302)
    for i in range(8):
        n = SLOT_LIMBS // 2 + i * 12345
        a, b = rand_limbs(rng, n), rand_limbs(rng, 3 * n // 4)
        if i % 3 == 1:
            a = pinned_like(a)
        c = bb.mul(a, b)
        assert port.mod_m61(a) * port.mod_m61(b) % M61 == port.mod_m61(c), i
