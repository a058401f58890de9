"""CPU model of the carry scan's decoupled look-back (the protocol of k_carry
in bigint_b200/csrc/ntt_kernels.cu), with host threads standing in for CTAs.

Each block owns a run of chunks, computes its (generate, propagate) pair,
publishes it as an aggregate flag, looks back over predecessors' flags until
one decides its carry-in (an inclusive flag, a generating aggregate or a
non-propagating aggregate), then publishes its inclusive flag.  Before that
it reads the `window` chunks below its run: when one of them does not
propagate, the highest such chunk's carry out is the block's carry-in and
no flag is waited on.  Checked against the serial carry of the same chunks in
random block orders, with runs of all-ones chunks that force long
look-backs; and a predecessor that never publishes makes the bounded wait
give up with an error, not hang."""
from __future__ import annotations

import random
import threading
import time

import pytest

MASK = (1 << 256) - 1


def serial_carries(chunks):
    out, c = [], 0
    for v in chunks:
        out.append(c)
        c = (v + c) >> 256
    return out


def block_gp(chunks):
    """(G, P) of a run: carry out with carry-in 0, and 'carry-in passes through'."""
    g, p = 0, 1
    for v in chunks:
        gi = v > MASK
        pi = (v & MASK) == MASK and not gi
        g = int(gi or (pi and g))
        p = int(p and pi)
    return g, p


def window_carry(chunks, start, window):
    """Carry into chunk `start` from the `window` chunks below it, or None
    when all of them propagate (k_carry's warp-0 read)."""
    for j in range(start - 1, start - window - 1, -1):
        if j < 0:
            return 0  # below chunk 0 nothing carries
        v = chunks[j]
        gi = v > MASK
        pi = (v & MASK) == MASK and not gi
        if not pi:
            return int(gi)
    return None


def run_protocol(chunks, per_block, order, stuck=None, spin_limit=200000, window=0):
    nblocks = (len(chunks) + per_block - 1) // per_block
    flags = [None] * nblocks  # (status, g, p): 1 aggregate, 2 inclusive
    err = []
    carry_in = [None] * nblocks
    lock = threading.Lock()

    def block(b):
        run = chunks[b * per_block:(b + 1) * per_block]
        g, p = block_gp(run)
        if b == stuck:
            return  # never publishes
        with lock:
            flags[b] = (2, g, 0) if b == 0 else (1, g, p)
        if b == 0:
            carry_in[0] = 0
            return
        if window:
            cin = window_carry(chunks, b * per_block, window)
            if cin is not None:
                carry_in[b] = cin
                with lock:
                    flags[b] = (2, g | (p & cin), 0)
                return
        k, cin, spins = b - 1, None, 0
        while True:
            with lock:
                f = flags[k]
            if f is None:
                spins += 1
                if spins > spin_limit:
                    err.append(b)
                    cin = 0
                    break
                time.sleep(0)
                continue
            st, fg, fp = f
            if st == 2:
                cin = fg
                break
            if fg:
                cin = 1
                break
            if not fp:
                cin = 0
                break
            k -= 1
        carry_in[b] = cin
        with lock:
            flags[b] = (2, g | (p & cin), 0)

    threads = [threading.Thread(target=block, args=(b,)) for b in order]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    return carry_in, err


def chunk_values(rng, n, ones_runs=()):
    vals = [rng.getrandbits(256) + rng.getrandbits(58) for _ in range(n)]  # chunk + spill
    for lo, hi in ones_runs:
        for i in range(lo, hi):
            vals[i] = MASK  # propagates any incoming carry
    return vals


@pytest.mark.parametrize("window", [0, 3, 32])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_lookback_matches_serial_carry(seed, window):
    rng = random.Random(seed)
    per_block = 4
    chunks = chunk_values(rng, 64, ones_runs=[(5, 30), (40, 41)])
    chunks[4] = MASK + 1  # a generate right before the long propagate run
    nblocks = len(chunks) // per_block
    order = list(range(nblocks))
    rng.shuffle(order)
    carry_in, err = run_protocol(chunks, per_block, order, window=window)
    assert not err
    want = serial_carries(chunks)
    for b in range(nblocks):
        assert carry_in[b] == want[b * per_block], b


def test_stuck_predecessor_times_out():
    rng = random.Random(7)
    chunks = chunk_values(rng, 16)
    carry_in, err = run_protocol(chunks, 4, [0, 1, 2, 3], stuck=1, spin_limit=2000)
    assert err == [2]  # block 2 waited on block 1, gave up and reported
    assert carry_in[0] == 0


def test_window_decides_without_flags_and_falls_back_on_long_runs():
    """The window alone decides every block of random chunks; a propagating run
    longer than the window sends the block above it to the flags."""
    rng = random.Random(11)
    chunks = chunk_values(rng, 64)
    want = serial_carries(chunks)
    for start in range(4, 64, 4):
        assert window_carry(chunks, start, 32) == want[start]
    chunks[10] = MASK + 5  # generates
    for i in range(11, 50):
        chunks[i] = MASK    # propagate
    assert window_carry(chunks, 50, 32) is None  # chunks 18..49 all propagate
    assert window_carry(chunks, 50, 48) == 1     # ... down to chunk 10, which generates
    carry_in, err = run_protocol(chunks, 2, list(range(32)), window=32)
    assert not err
    assert carry_in == [serial_carries(chunks)[b * 2] for b in range(32)]
