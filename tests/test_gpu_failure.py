"""Failure detection without a GPU fault: the carry scan's only wait is
bounded; here it runs (bgpu_selftest_wait) on a flag word that nothing sets,
gives up after a short limit, and reports BGPU_ERR_DEVICE_TIMEOUT through the
sticky device error word -- after which the context keeps working."""
from __future__ import annotations

import time

import numpy as np
import pytest

from conftest import SEED, rand_limbs

pytestmark = pytest.mark.gpu
BGPU_ERR_DEVICE_TIMEOUT = -7


def test_wait_on_unset_flag_times_out_and_context_survives(bb, port):
    t0 = time.perf_counter()
    assert bb.lib.bgpu_selftest_wait(20000, 0) == BGPU_ERR_DEVICE_TIMEOUT
    assert time.perf_counter() - t0 < 5.0  # gave up after its limit, well under a second typically
    assert bb.lib.bgpu_selftest_wait(20000, 1) == 0  # error word cleared; a set flag passes at once
    rng = np.random.default_rng(SEED + 80)
    a, b = rand_limbs(rng, 70000), rand_limbs(rng, 50000)
    assert np.array_equal(bb.mul(a, b), port.mul(a, b))  # tickets restarted, products still exact


def test_device_status_reports_and_clears(bb):
    assert bb.lib.bgpu_selftest_wait(1000, 0) == BGPU_ERR_DEVICE_TIMEOUT
    bb.device_status(0)  # nothing left to report


def test_concurrent_host_threads(bb, port):
    """The reference claims thread safety (README.md:10); calls from several
    host threads are serialized inside the library and each gets its own
    exact product."""
    import threading

    rng = np.random.default_rng(SEED + 81)
    jobs = [(rand_limbs(rng, n), rand_limbs(rng, m)) for n, m in
            [(5000, 4000), (100, 90), (70000, 1000), (3, 3), (20000, 20000), (128, 64)] * 3]
    want = [port.mul(a, b) for a, b in jobs]
    got = [None] * len(jobs)
    errors = []

    def worker(idx):
        try:
            for i in idx:
                got[i] = bb.mul(*jobs[i])
        except Exception as e:  # pragma: no cover - reported below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(range(t, len(jobs), 4),)) for t in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors
    for i, (g, w) in enumerate(zip(got, want)):
        assert np.array_equal(g, w), i


def test_concurrent_mixed_entry_points(bb, port):
    """Threads calling different entry points at once (u64 and Digits
    products through the staged host copies, the reciprocal, divmod, decimal
    parse and print, BigFloat print, fast_pow) share the engine's buffers; each
    result must equal the same call made alone."""
    import threading

    rng = np.random.default_rng(SEED + 82)
    a, b = rand_limbs(rng, 90000), rand_limbs(rng, 70000)
    d = rng.integers(0, 1 << 28, 150000, dtype=np.uint32)
    d[-1] |= 1
    text = "".join(map(str, rng.integers(0, 10, 60000)))
    na, nb, nf = d[:60000].copy(), d[:25000].copy(), d[:30000].copy()
    for x in (na, nb, nf):
        x[-1] |= 1  # no leading zero digit
    calls = [
        lambda: bb.mul(a, b),
        lambda: bb.mul_digits(d, d[:70000].copy()),
        lambda: bb.reciprocal_digits(d[:30000])[0],
        lambda: bb.from_decimal(text)[0],
        lambda: bb.to_decimal(d[:40000]),
        lambda: bb.fast_pow(7, 1000003),
        lambda: np.concatenate([x for (x, _) in bb.divmod_digits(na, nb, True, False, 1)]),
        lambda: bb.bigfloat_to_decimal(nf, 12000, False, 0),
    ]
    alone = [c() for c in calls]
    got = [[None] * len(calls) for _ in range(3)]
    errors = []

    def worker(r):
        try:
            for i in range(len(calls)):
                k = (i + r) % len(calls)
                got[r][k] = calls[k]()
        except Exception as e:  # pragma: no cover - reported below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(r,)) for r in range(3)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors
    for r in range(3):
        for k, want in enumerate(alone):
            g = got[r][k]
            assert (g == want) if isinstance(want, str) else np.array_equal(g, want), (r, k)
