"""Host-side logic of bench.py that needs no GPU: the byte models, the
operand-pair sizing, NVML clock-reason decoding against a fake NVML, and the
max-over-ranks reduction run as two gloo ranks on the CPU."""
from __future__ import annotations

import os
import socket
import sys
import types

import numpy as np
import pytest

import bench


def test_reference_model_bytes_matches_two_pass_formula():
    # 2^24 x 2^24 bits: N = 2^21 reference points, S = 12 N, B = 10 S + 2 (a+b)/8
    n = 1 << 18
    assert bench.reference_model_bytes(n, n) == 10 * 12 * (1 << 21) + 2 * 2 * n * 8
    assert bench.reference_model_bytes(n, n) == 260046848


def test_kernel_bytes_sum_for_headline():
    n = 1 << 18
    tot = sum(bench.kernel_bytes(k, n, n, 20, False)
              for k in ("k_fwd_cols", "k_mid_rows", "k_inv_cols", "k_carry"))
    s32 = 12 << 20
    assert tot == 6 * s32 + 2 * (5 << 20) + 2 * (2 * n * 8)


def test_pairs_exceed_l2():
    l2 = bench.l2_bytes()
    assert l2 >= 1 << 20
    for bits in (1 << 20, 1 << 24, 1 << 26):
        p = bench.pairs_beyond_l2(bits)
        assert p * 2 * bits // 8 >= 2 * l2 or p == 2


def test_make_operands_seeded_and_top_bit():
    a, b = bench.make_operands(1 << 12, pairs=3)
    a2, _ = bench.make_operands(1 << 12, pairs=3)
    assert np.array_equal(a, a2) and a.shape == (3, 64)
    assert np.all(a[:, -1] >> np.uint64(63) == 1) and np.all(b[:, -1] >> np.uint64(63) == 1)


def test_clock_sampler_decodes_reasons(monkeypatch):
    fake = types.SimpleNamespace(
        NVML_CLOCK_SM=0,
        nvmlClocksEventReasonSwPowerCap=0x4,
        nvmlClocksEventReasonHwSlowdown=0x8,
        nvmlClocksEventReasonHwThermalSlowdown=0x40,
        nvmlClocksEventReasonSwThermalSlowdown=0x20,
        nvmlInit=lambda: None,
        nvmlDeviceGetHandleByPciBusId=lambda s: "h",
        nvmlDeviceGetHandleByIndex=lambda i: "h",
        nvmlDeviceGetMaxClockInfo=lambda h, c: 1965,
    )
    seq = iter([(1800, 0x4), (1850, 0x4 | 0x1), (1900, 0x0)] + [(1900, 0)] * 10000)
    cur = {}

    def clock(h, c):
        cur["v"] = next(seq)
        return cur["v"][0]

    fake.nvmlDeviceGetClockInfo = clock
    fake.nvmlDeviceGetCurrentClocksEventReasons = lambda h: cur["v"][1]
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    import time

    with bench.ClockSampler("00000000:01:00.0", period=0.001) as clk:
        time.sleep(0.02)
    s = clk.summary()
    assert s["sm_max_mhz"] == 1965 and s["samples"] >= 3
    assert s["reasons"] == ["sw_power_cap"]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    v = bench.reduce_max(10.0 + rank, world)
    bench.barrier(world)
    q.put((rank, v))
    dist.destroy_process_group()


def test_reduce_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 11.0), (1, 11.0)]


def test_every_form_is_run_alone_and_in_the_default_run():
    """Each name in bench.FORMS is dispatched by --form and appears in the
    default run's "forms" object."""
    import inspect

    single = inspect.getsource(bench.run_single_form)
    default = inspect.getsource(bench.run_gpu_arm)
    missing = [name for name in bench.FORMS if f'"{name}"' not in single]
    assert missing in ([], [bench.FORMS[-1]])  # the last form is the dispatcher's final else
    for name in bench.FORMS:
        assert f'"{name}":' in default, name


def test_limb_digit_converters_round_trip():
    rng = np.random.default_rng(11)
    for n in (1, 2, 7, 64, 1001):
        limbs = rng.integers(0, 2**64, n, dtype=np.uint64)
        limbs[-1] |= np.uint64(1)
        d = bench.limbs_to_digits28_np(limbs)
        assert d.dtype == np.uint32 and int(d.max()) < (1 << 28) and d[-1] != 0
        assert sum(int(x) << (28 * i) for i, x in enumerate(d)) == int.from_bytes(limbs.tobytes(), "little")
        back = bench.digits28_to_limbs_np(d)
        assert np.array_equal(back[: n], limbs) and not back[n:].any()
