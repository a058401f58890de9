"""Benchmark: bit-exact big-integer products per second on one B200.

Workload (one step = one product): the plain three-prime NTT multiply of two
2^24-bit operands (262144 x 262144 u64 limbs), seeded uniform random limbs
with the top bit set -- the size the project's roofline target is stated at.
Inputs are generated on the host with a fixed seed and are synthetic.

Our arm (default):
  value      products/s with inputs resident in HBM (bgpu_mul_u64_device on a
             torch stream), K products back to back between two CUDA events;
             step i multiplies operand pair i mod P, where the P pairs together
             are larger than L2, so no step starts with its inputs cached.
  e2e        the same metric through the public host API from pinned host
             buffers: H2D of both operands, the kernels, D2H of the product,
             every step; bgpu_mul_u64_many pipelines the steps (copies overlap
             the multiplies), and the one-call-per-product figure
             (bgpu_mul_u64) is reported beside it (wall clock).
  roofline   dominant kernel of the pipeline: its algorithmic bytes per launch
             / its mean CUDA-event duration, against MEASURED_PEAKS.json.
  cpu_baseline  the reference's own CPU multiply (oracle/_ref, its thread
             pool at the host's core count) on a bounded sample, rank 0 only.
Reference arm (--impl reference): the reference CPU multiply on the host
cores for the same workload; rank 0 prints, other ranks exit.

Multi-GPU: products are independent, so N GPUs run N replicas ("replicas
only", weak scaling); times are the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

SEED = 0x9E3779B97F4A7C15
CONFIG_INDEX = 1  # the plain-NTT size sweep's 2^24-bit point
OPERAND_BITS = 1 << 24
L2_BYTES_B200 = 126 << 20  # B200's L2, when no device answers


def l2_bytes() -> int:
    """The device's L2 size (cudaDevAttrL2CacheSize, through torch's device
    properties), or B200's 126 MB without a device: the timed inputs of all
    operand pairs together must exceed it."""
    try:
        import torch

        if torch.cuda.is_available():
            n = int(getattr(torch.cuda.get_device_properties(torch.cuda.current_device()), "L2_cache_size", 0))
            if n > 0:
                return n
    except Exception:
        pass
    return L2_BYTES_B200


def make_operands(bits: int = OPERAND_BITS, seed: int = SEED + CONFIG_INDEX, pairs: int = 1):
    """`pairs` seeded operand pairs (uniform limbs, top bit set), as (pairs, n) arrays."""
    rng = np.random.default_rng(seed)
    n = bits // 64
    a = rng.integers(0, 2**64, (pairs, n), dtype=np.uint64, endpoint=False)
    b = rng.integers(0, 2**64, (pairs, n), dtype=np.uint64, endpoint=False)
    a[:, -1] |= np.uint64(1 << 63)
    b[:, -1] |= np.uint64(1 << 63)
    if pairs == 1:
        return a[0], b[0]
    return a, b


def pairs_beyond_l2(bits: int) -> int:
    """Distinct operand pairs whose inputs together are twice the L2 cache."""
    per_pair = 2 * bits // 8
    return max(2, -(-2 * l2_bytes() // per_pair))


def host_cores() -> int:
    """Logical CPUs this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def physical_cores() -> int:
    """Physical cores among the CPUs this process may run on (SMT siblings
    counted once), from the kernel's CPU topology; the logical count when the
    topology is not readable."""
    try:
        cpus = sorted(os.sched_getaffinity(0))
    except AttributeError:
        cpus = list(range(os.cpu_count() or 1))
    cores = set()
    for c in cpus:
        base = f"/sys/devices/system/cpu/cpu{c}/topology/"
        try:
            pkg = open(base + "physical_package_id").read().strip()
            core = open(base + "core_id").read().strip()
        except OSError:
            return len(cpus)
        cores.add((pkg, core))
    return max(1, len(cores))


def ref_pool_threads() -> int:
    """Thread count of the reference's pool inside this process (it is sized
    once per process): the physical cores, as the reference recommends."""
    return physical_cores()


def cpu_thread_counts() -> list[int]:
    """Thread counts the reference's CPU multiply is timed at: the physical
    cores (SMT siblings excluded, as the reference recommends for its pool),
    8 (the reference's own examples), and every logical CPU."""
    return sorted({physical_cores(), 8, host_cores()})


def workload_name(bits: int) -> str:
    return (f"plain three-prime NTT multiply, 2^{bits.bit_length() - 1} x 2^{bits.bit_length() - 1}"
            f"-bit operands ({bits // 64} x {bits // 64} u64 limbs), seeded uniform random limbs")


# ---- distributed helpers -------------------------------------------------------

def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def reduce_max(value: float, world: int, device=None) -> float:
    """Max of a per-rank float over all ranks (identity when world == 1)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int, device=None) -> None:
    if world > 1:
        import torch.distributed as dist

        if device is not None:
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


# ---- clocks sampling -------------------------------------------------------------

def pci_bus_id(device) -> str | None:
    """NVML-style PCI bus id ("00000000:1B:00.0") of a torch CUDA device."""
    import torch

    p = torch.cuda.get_device_properties(device)
    try:
        return f"{int(p.pci_domain_id):08X}:{int(p.pci_bus_id):02X}:{int(p.pci_device_id):02X}.0"
    except (AttributeError, TypeError, ValueError):
        return None


class ClockSampler:
    """Samples SM clock and clock-event reasons through NVML (the library
    nvidia-smi reads) every `period` seconds on a background thread while the
    timed region runs.  Read-only: no GPU setting is touched."""

    NAMES = {
        "nvmlClocksEventReasonSwPowerCap": "sw_power_cap",
        "nvmlClocksEventReasonHwSlowdown": "hw_slowdown",
        "nvmlClocksEventReasonHwThermalSlowdown": "hw_thermal_slowdown",
        "nvmlClocksEventReasonSwThermalSlowdown": "sw_thermal_slowdown",
        "nvmlClocksEventReasonHwPowerBrakeSlowdown": "hw_power_brake_slowdown",
        "nvmlClocksEventReasonSyncBoost": "sync_boost",
        "nvmlClocksEventReasonApplicationsClocksSetting": "applications_clocks_setting",
        "nvmlClocksEventReasonDisplayClockSetting": "display_clock_setting",
    }

    def __init__(self, pci_bus_id: str | None, period: float = 0.002):
        self.pci = pci_bus_id
        self.period = period
        self.samples: list[tuple[int, int]] = []
        self.smax = None
        self._stop = None
        self._thread = None
        self.error = None

    def __enter__(self):
        import threading

        try:
            import pynvml

            pynvml.nvmlInit()
            h = None
            if self.pci:
                try:
                    h = pynvml.nvmlDeviceGetHandleByPciBusId(self.pci)
                except Exception:
                    h = None
            if h is None:
                h = pynvml.nvmlDeviceGetHandleByIndex(0)
            self.smax = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            get_reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
            self._pynvml, self._h, self._get_reasons = pynvml, h, get_reasons
        except Exception as e:  # NVML missing: report unsampled
            self.error = repr(e)
            return self
        self._stop = threading.Event()

        def loop():
            while not self._stop.is_set():
                try:
                    sm = self._pynvml.nvmlDeviceGetClockInfo(self._h, self._pynvml.NVML_CLOCK_SM)
                    rs = int(self._get_reasons(self._h))
                    self.samples.append((sm, rs))
                except Exception as e:  # pragma: no cover
                    self.error = repr(e)
                    return
                self._stop.wait(self.period)

        self._thread = threading.Thread(target=loop, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.smax, "reasons": ["unsampled"],
                    "samples": 0, "source": "nvml", "error": self.error}
        reasons = set()
        for _, rs in self.samples:
            for attr, name in self.NAMES.items():
                bit = getattr(self._pynvml, attr, 0)
                if bit and rs & bit:
                    reasons.add(name)
        sm = [v for v, _ in self.samples]
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvml"}


# ---- roofline --------------------------------------------------------------------

def measured_peaks() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(path))["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def kernel_bytes(name: str, na: int, nb: int, log_n: int, square: bool) -> int:
    """Algorithmic global-memory bytes of one launch (minimal reads + writes)."""
    n = 1 << log_n
    s32 = 12 * n  # one operand's residues: 3 primes x u32 per point
    ops = 1 if square else 2
    inp = (na + (0 if square else nb)) * 8
    chunk_bytes = n // 2 * 8 + n // 8 * 8  # 256-bit chunk sums + spills
    return {
        "k_fwd_cols": inp + ops * s32,
        "k_mid_rows": ops * s32 + s32,
        "k_inv_cols": s32 + chunk_bytes,
        "k_carry": chunk_bytes + (na + nb) * 8,
    }[name]


def reference_model_bytes(na: int, nb: int) -> int:
    """Whole-product bytes of the two-pass NTT model pinned to the reference's
    28-bit digits: 10*S + 2*(a+b)/8 with S = 12*N, N = bit_ceil(da+db-1)."""
    da, db = -(-na * 64 // 28), -(-nb * 64 // 28)
    n = 1 << (da + db - 2).bit_length()
    return 10 * 12 * n + 2 * (na + nb) * 8


def _plan_rounds(l: int, maxr: int = 4) -> list[int]:
    """Radix round sizes of a length-2^l transform (the kernels' Plan<L>)."""
    nr = (l + maxr - 1) // maxr
    return [l // nr + (1 if k < l % nr else 0) for k in range(nr)]


def _bfly_muls(l: int) -> float:
    """32-bit multiply operations (mul.lo / mul.hi) of one length-2^l transform
    as the kernels run it: 3 per Shoup butterfly; butterflies whose twiddle is
    1 are skipped only in the round over the lowest bits."""
    r_last = _plan_rounds(l)[-1]
    stages = (l - r_last) + sum(1 - 2.0 ** -k for k in range(r_last))
    return (1 << (l - 1)) * stages * 3


def source_mul_counts(na: int, nb: int, log_n: int, log_n1: int, log_n2: int, square: bool) -> dict:
    """32-bit multiply operations per launch of each NTT kernel, counted from
    the kernels' source (butterflies x 3, Montgomery products x 3, the digit
    reduction x 2, Garner CRT x 14 per point); the compiler's own instruction
    choice (address arithmetic, moves on the multiply pipe) is not in it."""
    n, n1, n2 = 1 << log_n, 1 << log_n1, 1 << log_n2
    ops = 1 if square else 2
    half = 2 * 2 * max(na, nb) <= n  # every operand in the lower half: half the digits loaded
    loads = n // 2 if half else n
    fwd = ops * 3 * (n1 * _bfly_muls(log_n2) + 2 * loads + 6 * n + 4 * n // 8)
    r0 = _plan_rounds(log_n1)[0]
    mid = 3 * (n2 * (ops + 1) * _bfly_muls(log_n1) + 4 * n + 6 * n + 7 * n / (1 << r0))
    inv = 3 * n1 * _bfly_muls(log_n2) + 14 * n
    return {"k_fwd_cols": fwd, "k_mid_rows": mid, "k_inv_cols": inv, "k_carry": 0.0}


def profiled_pipes() -> dict | None:
    """Per-launch pipe counters of the four NTT kernels at 2^24 x 2^24 bits
    from the committed ncu summary, if any."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "ntt_2p24_pipes.json")))
    except (OSError, ValueError):
        return None


def compute_roofline(kernels_ms: dict, dom: str, prod_ms: float, sm_mhz: float | None, counts: dict) -> dict:
    """The ceiling that binds the transform passes: the 32-bit multiply pipe
    (fmaheavy: IMAD, IMAD.HI, IMAD.WIDE at 2 warp instructions per SM per
    cycle, the wide and high forms taking two of those slots) and instruction
    issue (4 warp instructions per SM per cycle).  Busy cycles per SM come
    from the committed ncu counters (a clock-independent count); the fraction
    divides them by the cycles of the live time at the sampled SM clock."""
    prof = profiled_pipes()
    res = {"bound": "int32 multiply pipe (fmaheavy)", "kernel": dom,
           "source_mul_ops_per_launch": counts.get(dom),
           "source_mul_ops_per_product": sum(counts.values()),
           "source_note": "counted from the kernel source: 3 per Shoup butterfly or Montgomery product, "
                          "2 per digit reduction, 14 per Garner CRT point"}
    if not prof or dom not in prof or not sm_mhz:
        res["profile"] = None
        return res
    clk = sm_mhz * 1e6
    k = prof[dom]
    live_cycles = kernels_ms[dom] * 1e-3 * clk
    res.update({
        "ncu_fmaheavy_warp_inst_per_launch": k["fmaheavy_warp_inst"],
        "ncu_thread_mul_inst_per_launch": k["fmaheavy_warp_inst"] * 32,
        "busy_cycles_per_sm": k["fmaheavy_busy_cycles_per_sm"],
        "achieved": k["fmaheavy_busy_cycles_per_sm"] / live_cycles,
        "peak": 1.0, "unit": "fraction of fmaheavy pipe cycles (sampled SM clock)",
        "frac": k["fmaheavy_busy_cycles_per_sm"] / live_cycles,
        "issue_frac": k["warp_inst"] / 148 / (4 * live_cycles),
        "ncu_busy_pct": k["fmaheavy_busy_pct"], "ncu_issue_active_pct": k["issue_active_pct"],
        "sm_mhz": sm_mhz,
    })
    names = [x for x in ("k_fwd_cols", "k_mid_rows", "k_inv_cols", "k_carry") if x in prof]
    busy = sum(prof[x]["fmaheavy_busy_cycles_per_sm"] for x in names)
    insts = sum(prof[x]["warp_inst"] for x in names)
    prod_cycles = prod_ms * 1e-3 * clk
    res["whole_product"] = {
        "busy_cycles_per_sm": busy, "cycles_per_product": prod_cycles,
        "frac": busy / prod_cycles, "issue_frac": insts / 148 / (4 * prod_cycles),
        "ncu_fmaheavy_warp_inst": sum(prof[x]["fmaheavy_warp_inst"] for x in names),
        "note": "all four kernels' multiply-pipe busy cycles per SM over the product time"}
    return res


def profiled_traffic(kernel: str) -> float | None:
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "ntt_2p24_traffic.json")
    try:
        return float(json.load(open(path))[kernel]["dram_bytes_per_launch"])
    except (OSError, KeyError, ValueError, TypeError):
        return None


# ---- CPU baseline ----------------------------------------------------------------

def cpu_reference_rate(a, b, seconds: float, max_reps: int, threads: int, min_reps: int = 1,
                       warmup: int = 1):
    """Products/s of the reference CPU multiply (or the C port when the
    reference library was not built), over a bounded sample: at least
    `min_reps` products and then until `seconds` or `max_reps`.  The
    reference's thread pool is sized once per process, so each thread count
    runs in a process of its own (`cpu_reference_rates`)."""
    from oracle.pyoracle import Port, Reference, have_reference

    if have_reference():
        impl, kind, cores = Reference(), "reference", threads
        impl.init_thread_pool(threads)
        fn = impl.mul
    else:
        impl, kind, cores = Port(), "port", 1
        fn = impl.ntt_mul
    fn(a[:1024], b[:1024])  # warm the pool
    for _ in range(max(1, warmup)):
        fn(a, b)  # and the full-size path: the reference's first large products run slower
    reps, t0 = 0, time.perf_counter()
    while True:
        fn(a, b)
        reps += 1
        el = time.perf_counter() - t0
        if reps >= min_reps and (el >= seconds or reps >= max_reps):
            break
    return reps / el, kind, cores, reps, el


def cpu_reference_rates(bits: int, seconds: float, max_reps: int, min_reps: int = 1,
                        warmup: int = 1) -> list[dict]:
    """`cpu_reference_rate` at every thread count of `cpu_thread_counts()`,
    each in a fresh process (the reference sizes its pool once per process).
    The pool's threads are the host's; nothing here touches a GPU."""
    import subprocess

    out = []
    for p in cpu_thread_counts():
        cmd = [sys.executable, os.path.abspath(__file__), "--cpu-worker", str(p), "--bits", str(bits),
               "--cpu-seconds", str(seconds), "--cpu-max-reps", str(max_reps),
               "--cpu-min-reps", str(min_reps), "--warmup", str(max(3, warmup))]
        env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
        r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1200)
        if r.returncode != 0:
            raise SystemExit(f"bench: CPU reference worker ({p} threads) failed: {r.stderr[-400:]}")
        out.append(json.loads(r.stdout.strip().splitlines()[-1]))
    return out


def run_cpu_worker(args) -> None:
    a, b = make_operands(args.bits)
    rate, kind, cores, reps, el = cpu_reference_rate(a, b, args.cpu_seconds, args.cpu_max_reps, args.cpu_worker,
                                                     min_reps=args.cpu_min_reps, warmup=args.warmup)
    print(json.dumps({"threads": cores, "kind": kind, "rate": rate, "reps": reps, "seconds": el}))


# ---- the other configurations, reported beside the headline -----------------------

def _dev_limbs(torch, device, x):
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int64)).to(device)


def _event_ms(torch, stream, fn, reps):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for i in range(reps):
            fn(i)
        e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def plain_2p20_form(bb, torch, device, port, cpu: bool = True):
    """Config "plain NTT, 2^20 x 2^20": one product of two seeded uniform
    2^20-bit operands (16384 limbs each, top bit set), device resident (CUDA
    events, one product at a time) and through the host API
    (bgpu_mul_u64, pageable buffers, wall clock), compared limb-exact with the
    reference's ntt::mul (src/mul/ntt_multithread.cpp:444), which is timed on
    the host cores beside it."""
    rng = np.random.default_rng(SEED + 1)
    n = (1 << 20) // 64
    a = rng.integers(0, 2**64, n, dtype=np.uint64)
    b = rng.integers(0, 2**64, n, dtype=np.uint64)
    a[-1] |= np.uint64(1 << 63)
    b[-1] |= np.uint64(1 << 63)
    stream = torch.cuda.Stream(device)
    sp = stream.cuda_stream
    da, db = _dev_limbs(torch, device, a), _dev_limbs(torch, device, b)
    out = torch.empty(2 * n, dtype=torch.int64, device=device)

    def run(i):
        bb.mul_device(da.data_ptr(), n, db.data_ptr(), n, out.data_ptr(), stream=sp,
                      method=bb.BGPU_METHOD_NTT)
    run(0)
    bb.device_status(sp)
    dev_ms = _event_ms(torch, stream, run, 50)
    bb.device_status(sp)
    got_dev = out.cpu().numpy().view(np.uint64)
    bb.mul(a, b)
    t0 = time.perf_counter()
    for _ in range(20):
        got = bb.mul(a, b)
    host_ms = (time.perf_counter() - t0) / 20 * 1e3
    res = {"a_bits": 1 << 20, "b_bits": 1 << 20, "device_ms": dev_ms, "host_api_ms": host_ms,
           "products_per_s": 1e3 / dev_ms}
    from oracle.pyoracle import Reference, have_reference

    if have_reference():
        ref = Reference()
        ref.init_thread_pool(ref_pool_threads())
        for _ in range(3):  # the pool's threads and first-touch pages warm up over the first calls
            want = ref.ntt_mul(a, b)
        if cpu:
            ts = []
            for _ in range(7):
                t0 = time.perf_counter()
                ref.ntt_mul(a, b)
                ts.append(time.perf_counter() - t0)
            res["cpu_reference"] = {"ms": statistics.median(ts) * 1e3, "threads": ref_pool_threads(),
                                    "call": "bigint::mul::ntt::mul (median of 7 after 3 warm-up calls)"}
        res["verified"] = "limb-exact vs the reference's ntt::mul"
    else:
        want = port.ntt_mul(a, b)
        res["verified"] = "limb-exact vs the C restatement"
    if not (np.array_equal(got, want) and np.array_equal(got_dev[: want.size], want)):
        raise SystemExit("bench plain 2^20: product differs from the reference")
    return res


def sweep_form(bb, torch, device, port):
    """Config "NTT size sweep": squares at 2^16..2^30 bits, uniform and all-ones
    limbs, plus the 1:8 and 1:64 unbalanced pairs, and two sizes beyond the
    largest transform (2^31 x 2^31 bits, a 2^32-bit square: spectral sums of
    block products);
    device-resident products back to back on one stream (operands smaller
    than L2 stay cached there)."""
    stream = torch.cuda.Stream(device)
    sp = stream.cuda_stream
    M = (1 << 61) - 1
    rng = np.random.default_rng(SEED + 2)
    rows = []
    from oracle.pyoracle import Reference, have_reference

    ref = None
    if have_reference():  # products up to 2^27 bits also limb-exact vs ntt::mul (at most ~1 s each)
        ref = Reference()
        ref.init_thread_pool(ref_pool_threads())
    cases = [(1 << b, 1 << b, "square") for b in range(16, 31, 2)]
    cases += [(1 << 24, 1 << 21, "1:8"), (1 << 20, 1 << 14, "1:64")]
    # beyond the largest transform (2^31 product bits): 2^30-bit blocks, each
    # transformed once, output blocks formed as spectral sums
    cases += [(1 << 31, 1 << 31, "1:1"), (1 << 32, 1 << 32, "square")]
    for abits, bbits, kind in cases:
        na, nb = abits // 64, bbits // 64
        for fill in ("uniform", "all-ones"):
            if fill == "uniform":
                a = rng.integers(0, 2**64, na, dtype=np.uint64, endpoint=False)
                a[-1] |= np.uint64(1 << 63)
                b = a if kind == "square" else rng.integers(0, 2**64, nb, dtype=np.uint64, endpoint=False)
                if kind != "square":
                    b[-1] |= np.uint64(1 << 63)
            else:
                a = np.full(na, np.uint64(0xFFFFFFFFFFFFFFFF))
                b = a if kind == "square" else np.full(nb, np.uint64(0xFFFFFFFFFFFFFFFF))
            da = _dev_limbs(torch, device, a)
            db = da if kind == "square" else _dev_limbs(torch, device, b)
            out = torch.empty(na + nb, dtype=torch.int64, device=device)

            def run(i):
                bb.mul_device(da.data_ptr(), na, db.data_ptr(), nb, out.data_ptr(), stream=sp,
                              method=bb.BGPU_METHOD_NTT)
            reps = 3 if abits >= 1 << 28 else 20
            if abits >= 1 << 31:
                reps = 2
            run(0)
            bb.device_status(sp)
            ms = _event_ms(torch, stream, run, reps)
            bb.device_status(sp)
            c = out.cpu().numpy().view(np.uint64)
            ok = port.mod_m61(a) * port.mod_m61(b) % M == port.mod_m61(c)
            if not ok:
                raise SystemExit(f"bench sweep: residue check failed at {abits}x{bbits} {fill}")
            verified = "residue mod 2^61-1"
            if ref is not None and abits + bbits <= 1 << 27:
                want = ref.ntt_mul(a) if kind == "square" else ref.ntt_mul(a, b)
                if not np.array_equal(np.trim_zeros(c, "b"), want):
                    raise SystemExit(f"bench sweep: {abits}x{bbits} {fill} differs from the reference's ntt::mul")
                verified += "; limb-exact vs the reference's ntt::mul"
            model = reference_model_bytes(na, nb)
            rows.append({"a_bits": abits, "b_bits": bbits, "kind": kind, "limbs": fill,
                         "ms": ms, "products_per_s": 1e3 / ms,
                         "log2_points": (2 * na + 2 * nb - 2).bit_length(),
                         "reference_model_frac": model / (ms * 1e-3) / 1e9 / measured_peaks()[0],
                         "verified": verified})
            del da, db, out
    return rows


def fft_form(bb, torch, device, reps: int = 3):
    """Config "FP64 FFT vs NTT": the FFT form at 2^20..2^28-bit operands,
    uniform products and all-ones squares, bits per point from the worst-case
    and from the average error bound; device time of the FFT kernels per
    product (events inside the host call), the measured max rounding distance,
    whether the product was recomputed on the NTT, and the NTT's device time
    for the same operands.  Sizes beyond the FFT's capacity (its transform
    length or the FP64 coefficient limit) run on the NTT and say so."""
    rng = np.random.default_rng(SEED + 4)
    rows = []
    from oracle.pyoracle import Reference, have_reference

    ref = None
    if have_reference():
        ref = Reference()
        ref.init_thread_pool(ref_pool_threads())
    for k in (20, 22, 24, 26, 28):
        n = (1 << k) // 64
        a = rng.integers(0, 2**64, n, dtype=np.uint64, endpoint=False)
        b = rng.integers(0, 2**64, n, dtype=np.uint64, endpoint=False)
        a[-1] |= np.uint64(1 << 63)
        b[-1] |= np.uint64(1 << 63)
        ones = np.full(n, np.uint64(0xFFFFFFFFFFFFFFFF))
        for fill, x, y in (("uniform", a, b), ("all-ones", ones, None)):
            args = (x,) if y is None else (x, y)
            nt = [bb.ntt_mul(*args, stats=True) for _ in range(reps + 1)]
            want = nt[-1][0]
            verified = "identical to the NTT product"
            if ref is not None and k <= 24:
                if not np.array_equal(want, ref.mul(*args)):
                    raise SystemExit(f"bench fft: NTT product at 2^{k} bits differs from the reference's _mul")
                verified = "identical to the NTT product and to the reference's _mul"
            for bound, avg in (("worst_case", False), ("average", True)):
                runs = [bb.fft_mul(*args, average_bound=avg, stats=True) for _ in range(reps + 1)][1:]
                sts = [r[1] for r in runs]
                if not all(np.array_equal(r[0], want) for r in runs):
                    raise SystemExit(f"bench fft: FFT-form product at 2^{k} bits ({fill}, {bound}) is not exact")
                st = sts[-1]
                used = "ntt (fallback)" if st.fell_back else (
                    "fft" if st.method == bb.BGPU_METHOD_FFT else "ntt (beyond fft capacity)")
                rows.append({"operand_bits": 1 << k, "limbs": fill, "bound": bound,
                             "bits_per_point": st.fft_bits or None, "log2_points": st.log2_points,
                             "method": used, "max_round_err": st.max_round_err,
                             "fell_back": bool(st.fell_back),
                             "fallbacks": sum(1 for s_ in sts if s_.fell_back), "runs": len(sts),
                             "device_ms": statistics.fmean(s_.device_ms for s_ in sts),
                             "ntt_device_ms": statistics.fmean(r[1].device_ms for r in nt[1:]),
                             "verified": verified})
    return rows


def mul_digits_form(bb, port, cpu: bool = True, reps: int = 20):
    """The reference's main seam at the headline size: mul_digits on 28-bit
    Digits (BigInt::operator*, include/bigint/bigint.h:289) of two 2^24-bit
    numbers (599187 digits each) through the host API bgpu_mul_digits (H2D
    of both operands, the kernels reading and writing Digits directly, D2H of
    the product), wall clock; the reference's own mul_digits on the host cores
    beside it (one run)."""
    rng = np.random.default_rng(SEED + 6)
    nd = -(-(1 << 24) // 28)
    top = (1 << 24) - 28 * (nd - 1)  # bits in the top digit: exactly 2^24 bits in all
    a = rng.integers(0, 1 << 28, nd, dtype=np.uint32)
    b = rng.integers(0, 1 << 28, nd, dtype=np.uint32)
    for x in (a, b):
        x[-1] = (x[-1] & np.uint32((1 << top) - 1)) | np.uint32(1 << (top - 1))
    bb.mul_digits(a, b)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        got = bb.mul_digits(a, b)
        times.append(time.perf_counter() - t0)
    el = statistics.median(times)
    res = {"digits_per_operand": nd, "ms": el * 1e3, "mean_ms": sum(times) / reps * 1e3,
           "products_per_s": 1.0 / el, "api": "bgpu_mul_digits (host buffers, median of 20 calls)"}
    from oracle.pyoracle import Reference, have_reference

    if cpu and have_reference():
        ref = Reference()
        ref.init_thread_pool(ref_pool_threads())
        t0 = time.perf_counter()
        want = ref.mul_digits(a, b)
        res["cpu_reference"] = {"s": time.perf_counter() - t0, "threads": ref_pool_threads(),
                                "call": "bigint::mul::mul_digits"}
        if not np.array_equal(got, want):
            raise SystemExit("bench mul_digits: product differs from the reference")
        res["verified"] = "identical to the reference's mul_digits"
    else:
        M = (1 << 61) - 1
        if port.mod_m61(digits28_to_limbs_np(a)) * port.mod_m61(digits28_to_limbs_np(b)) % M != \
                port.mod_m61(digits28_to_limbs_np(got)):
            raise SystemExit("bench mul_digits: residue check failed")
        res["verified"] = "residue mod 2^61-1"
    return res


def digits28_to_limbs_np(d) -> np.ndarray:
    """Little-endian 28-bit digits -> u64 limbs (vectorised bit repacking)."""
    d = np.ascontiguousarray(d, dtype=np.uint32)
    bits = np.unpackbits(d.view(np.uint8), bitorder="little").reshape(-1, 32)[:, :28].ravel()
    pad = (-bits.size) % 64
    if pad:
        bits = np.concatenate([bits, np.zeros(pad, dtype=np.uint8)])
    limbs = np.packbits(bits, bitorder="little").view(np.uint64)
    n = limbs.size
    while n and limbs[n - 1] == 0:
        n -= 1
    return limbs[:n]


def fast_pow_form(bb, port, cpu: bool = True):
    """The reference's benchmark call fast_pow(1234567, 7654321)
    (examples/benchmark.cpp:22): the whole squaring chain on the GPU through
    the host API, wall clock, residue-checked; the reference's own fast_pow on
    the host cores beside it (one run)."""
    base, e = 1234567, 7654321
    bb.fast_pow(base, 1001)  # warm-up
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        got = bb.fast_pow(base, e)
        times.append(time.perf_counter() - t0)
    m = (1 << 61) - 1
    if port.mod_m61(got) != pow(base, e, m):
        raise SystemExit("bench fast_pow: residue check failed")
    res = {"call": "fast_pow(1234567, 7654321)", "result_bits": int(got.size * 64),
           "s": statistics.median(times), "launches": bb.last_launch_count(),
           "verified": "residue mod 2^61-1"}
    from oracle.pyoracle import REF_GPU_SO, Reference, have_reference, have_reference_gpu

    if have_reference_gpu():
        # the reference's own fast_pow<BigInt> (unmodified C++), its products
        # hooked to this engine (bigint_b200/hooks/reference_hook.cpp)
        hooked = Reference(REF_GPU_SO)
        hooked.init_thread_pool(1)
        hooked.fast_pow_digits(base, 1001)
        t0 = time.perf_counter()
        d = hooked.fast_pow_digits(base, e)
        el = time.perf_counter() - t0
        same = np.array_equal(digits28_to_limbs_np(d), got)
        if not same:
            raise SystemExit("bench fast_pow: hooked reference differs from bgpu_pow_u64")
        res["reference_code_on_gpu"] = {"s": el, "call": "bigint::fast_pow<BigInt> with ntt::mul and "
                                        "fft::mul hooked to bgpu_mul_u64", "identical": same}
    if have_reference() and Reference().has_fast_pow:
        ref = Reference()
        ref.init_thread_pool(ref_pool_threads())
        t0 = time.perf_counter()
        want = ref.fast_pow_digits(base, e)
        t_ref = time.perf_counter() - t0
        if not np.array_equal(digits28_to_limbs_np(want), got):
            raise SystemExit("bench fast_pow: bgpu_pow_u64 differs from the reference's fast_pow")
        res["verified"] += "; identical to the reference's fast_pow<BigInt>"
        if cpu:
            res["cpu_reference"] = {"s": t_ref, "threads": ref_pool_threads(),
                                    "call": "bigint::fast_pow<BigInt>"}
    return res


def reciprocal_form(bb, cpu: bool = True, reps: int = 5):
    """BigFloat::reciprocal (src/bigint.cpp:1044-1071) of a 2^24-bit value at
    its own precision (599187 digits) through bgpu_reciprocal_digits, every
    Newton step on the device, wall clock from host Digits to host Digits;
    the reference's own reciprocal on the host cores beside it (one run),
    digits, point and sign compared."""
    rng = np.random.default_rng(SEED + 7)
    limbs = rng.integers(0, 2**64, (1 << 24) // 64, dtype=np.uint64)
    limbs[-1] |= np.uint64(1 << 63)
    digits = limbs_to_digits28_np(limbs)
    tz = int(np.argmax(digits != 0))  # BigFloat(BigInt) drops bottom zero digits
    digits, pp_in = digits[tz:], -tz
    bb.reciprocal_digits(digits, pp_in)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        got, pp, neg = bb.reciprocal_digits(digits, pp_in)
        times.append(time.perf_counter() - t0)
    res = {"input_bits": 1 << 24, "precision_digits": int(digits.size), "result_digits": int(got.size),
           "s": statistics.median(times), "api": "bgpu_reciprocal_digits (host Digits in and out)"}
    from oracle.pyoracle import Reference, have_reference

    if cpu and have_reference() and Reference().has_bigfloat_reciprocal:
        ref = Reference()
        ref.init_thread_pool(ref_pool_threads())
        t0 = time.perf_counter()
        (din, ppin, _), (want, wpp, wneg) = ref.bigfloat_reciprocal(limbs, 0, False, 0)
        res["cpu_reference"] = {"s": time.perf_counter() - t0, "threads": ref_pool_threads(),
                                "call": "BigFloat::reciprocal"}
        if not (np.array_equal(din, digits) and ppin == pp_in and np.array_equal(got, want) and pp == wpp
                and neg == wneg):
            raise SystemExit("bench reciprocal: result differs from the reference's")
        res["verified"] = "identical to the reference's reciprocal"
    else:
        # x * r within 2^(-28 k) of 1 for k = half the precision (Newton's
        # previous step alone guarantees that much)
        prod = bb.mul_digits(digits, got)  # point position pp_in + pp
        k = digits.size // 2
        top = prod[pp_in + pp - k:]
        t = int.from_bytes(digits28_to_limbs_np(top).tobytes(), "little")
        if t not in ((1 << (28 * k)) - 1, 1 << (28 * k)):
            raise SystemExit("bench reciprocal: x * (1/x) is not close to 1")
        res["verified"] = f"x * (1/x) = 1 to {28 * k} bits"
    return res


def divmod_form(bb, port, cpu: bool = True, reps: int = 5):
    """BigInt::divmod (src/bigint.cpp:625-673) of a 2^24-bit integer by a
    2^23-bit one, truncating, through bgpu_divmod_digits: the reciprocal at
    n_a + 16 digits, the estimate, Q * b and the check all on the device, wall
    clock from host Digits to host Digits; the reference's own divmod on the
    host cores beside it (one run), quotient and remainder compared."""
    rng = np.random.default_rng(SEED + 10)
    la = rng.integers(0, 2**64, (1 << 24) // 64, dtype=np.uint64)
    lb = rng.integers(0, 2**64, (1 << 23) // 64, dtype=np.uint64)
    la[-1] |= np.uint64(1 << 63)
    lb[-1] |= np.uint64(1 << 63)
    a, b = limbs_to_digits28_np(la), limbs_to_digits28_np(lb)
    bb.divmod_digits(a, b)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        (q, qn), (r, rn) = bb.divmod_digits(a, b)
        times.append(time.perf_counter() - t0)
    res = {"a_bits": 1 << 24, "b_bits": 1 << 23, "mode": "Truncate", "quotient_digits": int(q.size),
           "s": statistics.median(times), "api": "bgpu_divmod_digits (host Digits in and out)"}
    from oracle.pyoracle import Reference, have_reference

    if cpu and have_reference() and Reference().has_divmod:
        ref = Reference()
        ref.init_thread_pool(ref_pool_threads())
        t0 = time.perf_counter()
        (wq, wqn), (wr, wrn) = ref.divmod(la, False, lb, False, 0, True)
        res["cpu_reference"] = {"s": time.perf_counter() - t0, "threads": ref_pool_threads(),
                                "call": "BigInt::divmod"}
        if not (np.array_equal(q, wq) and qn == wqn and np.array_equal(r, wr) and rn == wrn):
            raise SystemExit("bench divmod: result differs from the reference's")
        res["verified"] = "identical to the reference's quotient and remainder"
    else:
        m61 = (1 << 61) - 1
        lq, lr = digits28_to_limbs_np(q), digits28_to_limbs_np(r)
        if (port.mod_m61(lq) * port.mod_m61(lb) + port.mod_m61(lr)) % m61 != port.mod_m61(la) or qn or rn:
            raise SystemExit("bench divmod: A != Q * B + R")
        if r.size > b.size or (r.size == b.size and r[::-1].tolist() >= b[::-1].tolist()):
            raise SystemExit("bench divmod: remainder not below the divisor")
        res["verified"] = "A = Q * B + R mod 2^61 - 1 and 0 <= R < B"
    return res


def bigfloat_print_form(bb, cpu: bool = True, reps: int = 5):
    """BigFloat::print (src/bigint.cpp:972-1041) of a 2^22-bit value with the
    point in the middle and the default fraction length (all its fraction
    Digits: 631 306 decimals), through bgpu_bigfloat_to_decimal (5^d, the
    scaled fraction, its rounding and both decimal conversions on the device);
    the reference's own print on the host cores beside it (one run), texts
    compared."""
    rng = np.random.default_rng(SEED + 11)
    limbs = rng.integers(0, 2**64, (1 << 22) // 64, dtype=np.uint64)
    limbs[-1] |= np.uint64(1 << 63)
    limbs[0] |= np.uint64(1)  # no zero digit at the bottom: the fields below are BigFloat(X, offset)'s
    digits = limbs_to_digits28_np(limbs)
    offset = -28 * (digits.size // 2)
    pp = digits.size // 2
    bb.bigfloat_to_decimal(digits, pp)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        text = bb.bigfloat_to_decimal(digits, pp)
        times.append(time.perf_counter() - t0)
    res = {"bits": 1 << 22, "point_pos": pp, "chars": len(text), "s": statistics.median(times),
           "api": "bgpu_bigfloat_to_decimal (host Digits in, host text out)"}
    from oracle.pyoracle import Reference, have_reference

    if cpu and have_reference() and Reference().has_bigfloat_print:
        ref = Reference()
        ref.init_thread_pool(ref_pool_threads())
        t0 = time.perf_counter()
        (din, ppin), want = ref.bigfloat_print(limbs, offset, False, 0)
        res["cpu_reference"] = {"s": time.perf_counter() - t0, "threads": ref_pool_threads(),
                                "call": "BigFloat::print"}
        if not (np.array_equal(din, digits) and ppin == pp and text == want):
            raise SystemExit("bench BigFloat print: text differs from the reference's")
        res["verified"] = "identical text"
    else:
        head, frac = text.split(".")
        if bb.to_decimal(digits[pp:]) != head or len(frac) != int(28 * pp * 0.30102999566398120):
            raise SystemExit("bench BigFloat print: integer part or fraction length wrong")
        res["verified"] = "integer part equals bgpu_to_decimal's; fraction length"
    return res


def decimal_print_form(bb, cpu: bool = True):
    """Decimal text of a 2^22-bit integer (1.26 M digits): bgpu_to_decimal
    (the whole conversion on the GPU, host Digits in, host text out); the
    reference's own BigInt::print (src/bigint.cpp:175-247: print_dec's divide
    and conquer over get_pow_of_ten and divmod), unmodified C++, with its
    products hooked to this engine (bigint_b200/hooks/reference_hook.cpp); and
    the same code on the host cores alone.  All three strings compared."""
    from oracle.pyoracle import REF_GPU_SO, Reference, have_reference, have_reference_gpu

    rng = np.random.default_rng(SEED + 8)
    limbs = rng.integers(0, 2**64, (1 << 22) // 64, dtype=np.uint64)
    limbs[-1] |= np.uint64(1 << 63)
    digits = limbs_to_digits28_np(limbs)
    bb.to_decimal(digits[:1000])  # small warm-up: the engine's power cache covers small sizes only
    t0 = time.perf_counter()
    s_native = bb.to_decimal(digits)
    first = time.perf_counter() - t0  # includes growing the cache of 10^(19*2^k) and reciprocals
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        s_native = bb.to_decimal(digits)
        times.append(time.perf_counter() - t0)
    res = {"input_bits": 1 << 22, "decimal_digits": len(s_native), "s": statistics.median(times),
           "first_call_s": first, "api": "bgpu_to_decimal",
           "note": "s: repeated calls (powers of ten cached, as the reference caches them); "
                   "first_call_s: the first call at this size, which builds them"}
    # a 46.6 M-digit number (2,418,800 limbs), printed and parsed back on the
    # GPU; the reference's decimal conversion takes minutes at this size, so
    # each direction is checked against it at the size above and in the tests
    big = rng.integers(0, 2**64, 2_418_800, dtype=np.uint64)
    big[-1] |= np.uint64(1 << 63)
    big_digits = limbs_to_digits28_np(big)
    bb.to_decimal(big_digits)
    t0 = time.perf_counter()
    text = bb.to_decimal(big_digits)
    t_print = time.perf_counter() - t0
    t0 = time.perf_counter()
    back, _ = bb.from_decimal(text)
    t_parse = time.perf_counter() - t0
    if not np.array_equal(back, big_digits):
        raise SystemExit("bench decimal: 46.6 M-digit round trip differs")
    res["large"] = {"input_bits": int(big.size * 64), "decimal_digits": len(text), "to_decimal_s": t_print,
                    "from_decimal_s": t_parse, "verified": "round trip identical"}
    if not have_reference_gpu():
        return res
    hooked = Reference(REF_GPU_SO)
    hooked.init_thread_pool(1)
    if not hooked.has_to_dec:
        return {"unavailable": "reference shim without ref_to_dec_string"}
    hooked.to_dec_string(limbs[:4096])
    t0 = time.perf_counter()
    s_gpu = hooked.to_dec_string(limbs)
    res["reference_code_on_gpu"] = {"s": time.perf_counter() - t0,
                                    "call": "BigInt::print with ntt::mul / fft::mul hooked to bgpu_mul_u64"}
    if s_gpu != s_native:
        raise SystemExit("bench decimal: bgpu_to_decimal and the hooked reference print different text")
    if cpu and have_reference():
        ref = Reference()
        ref.init_thread_pool(ref_pool_threads())
        ref.to_dec_string(limbs[:4096])
        t0 = time.perf_counter()
        s_cpu = ref.to_dec_string(limbs)
        res["cpu_reference"] = {"s": time.perf_counter() - t0, "threads": ref_pool_threads(), "call": "BigInt::print"}
        if s_cpu != s_gpu:
            raise SystemExit("bench decimal: hooked reference prints a different number")
        res["verified"] = "identical decimal text (native, hooked reference, pure reference)"
    return res


def decimal_parse_form(bb, cpu: bool = True):
    """Decimal text of 5 M digits (about 2^24 bits) to a BigInt: the
    reference's BigInt(const std::string&) (src/bigint.cpp:25-124) on the
    host cores beside bgpu_from_decimal (leaves and level products on the
    GPU), host text in and host Digits out, results compared."""
    rng = np.random.default_rng(SEED + 9)
    d = rng.integers(0, 10, 5_000_000, dtype=np.uint8)
    d[0] = 4
    text = (d + ord("0")).tobytes()
    bb.from_decimal(text[:100000])  # small warm-up: the engine's power cache covers small sizes only
    t0 = time.perf_counter()
    got, neg = bb.from_decimal(text)
    first = time.perf_counter() - t0  # includes growing the cache of 10^(19*2^k)
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        got, neg = bb.from_decimal(text)
        times.append(time.perf_counter() - t0)
    res = {"decimal_digits": len(text), "s": statistics.median(times), "first_call_s": first,
           "api": "bgpu_from_decimal"}
    from oracle.pyoracle import Reference, have_reference

    if have_reference() and Reference().has_from_dec:
        ref = Reference()
        ref.init_thread_pool(ref_pool_threads())
        ref.from_dec_string(text[:100000])
        if cpu:
            t0 = time.perf_counter()
        want, wneg = ref.from_dec_string(text)
        if cpu:
            res["cpu_reference"] = {"s": time.perf_counter() - t0, "threads": ref_pool_threads(),
                                    "call": "BigInt(const std::string&)"}
        if not (np.array_equal(got, want) and neg == wneg):
            raise SystemExit("bench decimal parse: result differs from the reference's")
        res["verified"] = "identical Digits"
    return res


def limbs_to_digits28_np(limbs) -> np.ndarray:
    """u64 limbs -> little-endian 28-bit digits without leading zeros."""
    bits = np.unpackbits(np.ascontiguousarray(limbs, dtype=np.uint64).view(np.uint8), bitorder="little")
    pad = (-bits.size) % 28
    if pad:
        bits = np.concatenate([bits, np.zeros(pad, dtype=np.uint8)])
    b = bits.reshape(-1, 28)
    d = np.zeros(b.shape[0], dtype=np.uint32)
    for k in range(28):
        d |= b[:, k].astype(np.uint32) << np.uint32(k)
    n = d.size
    while n > 1 and d[n - 1] == 0:
        n -= 1
    return d[:n]


BATCH_SEED = SEED + 3


def batched_sizes(nprod: int = 4096, seed: int = BATCH_SEED):
    """Operand lengths (u64 limbs) of the batched uneven workload: each
    operand's bit length log-uniform in [2^10, 2^22], drawn independently."""
    rng = np.random.default_rng(seed)
    na = np.maximum(1, (np.exp2(rng.uniform(10, 22, nprod)) // 64).astype(np.int64))
    nb = np.maximum(1, (np.exp2(rng.uniform(10, 22, nprod)) // 64).astype(np.int64))
    return na, nb


def batched_operands(i: int, na: int, nb: int, seed: int = BATCH_SEED):
    """Operands of product i of the batched workload: uniform limbs, top bit
    set, from a stream of their own (so any product can be rebuilt alone)."""
    rng = np.random.default_rng([seed, i])
    a = rng.integers(0, 2**64, int(na), dtype=np.uint64, endpoint=False)
    b = rng.integers(0, 2**64, int(nb), dtype=np.uint64, endpoint=False)
    a[-1] |= np.uint64(1 << 63)
    b[-1] |= np.uint64(1 << 63)
    return a, b


def batched_inputs(nprod: int = 4096, seed: int = BATCH_SEED):
    """The whole batched workload in one array: (big, offs_a, na, offs_b, nb)."""
    na, nb = batched_sizes(nprod, seed)
    offs_a = np.concatenate([[0], np.cumsum(na)[:-1]])
    offs_b = np.concatenate([[0], np.cumsum(nb)[:-1]]) + na.sum()
    big = np.empty(int(na.sum() + nb.sum()), dtype=np.uint64)
    for i in range(nprod):
        a, b = batched_operands(i, na[i], nb[i], seed)
        big[offs_a[i]:offs_a[i] + na[i]] = a
        big[offs_b[i]:offs_b[i] + nb[i]] = b
    return big, offs_a, na, offs_b, nb


def batched_form(bb, torch, device, port, nprod: int = 4096, runs: int = 5, ref_every: int = 64):
    """Config "batched uneven": 4096 products, operand lengths log-uniform in
    [2^10, 2^22] bits, one graph launch per batch vs one plain NTT call per
    product (same inputs, device resident, > L2 in total).  Every product is
    checked by its residue and against the one-call-per-product output; every
    `ref_every`-th product also limb-exact against the reference's _mul."""
    big, offs_a, na, offs_b, nb = batched_inputs(nprod)
    dbig = _dev_limbs(torch, device, big)
    outn = na + nb
    offs_o = np.concatenate([[0], np.cumsum(outn)[:-1]])
    dout = torch.zeros(int(outn.sum()), dtype=torch.int64, device=device)
    base_in, base_out = dbig.data_ptr(), dout.data_ptr()
    prods = [(base_in + 8 * int(offs_a[i]), int(na[i]), base_in + 8 * int(offs_b[i]), int(nb[i]),
              base_out + 8 * int(offs_o[i])) for i in range(nprod)]
    t_plan = time.perf_counter()
    plan = bb.BatchPlan(prods)
    t_plan = time.perf_counter() - t_plan
    stream = torch.cuda.Stream(device)
    sp = stream.cuda_stream
    for _ in range(2):
        plan.run(sp)
    bb.device_status(sp)
    ms_batch = _event_ms(torch, stream, lambda i: plan.run(sp), runs)
    bb.device_status(sp)
    host = dout.cpu().numpy().view(np.uint64)
    M = (1 << 61) - 1
    for i in range(nprod):
        a = big[offs_a[i]:offs_a[i] + na[i]]
        b = big[offs_b[i]:offs_b[i] + nb[i]]
        c = host[offs_o[i]:offs_o[i] + outn[i]]
        if port.mod_m61(a) * port.mod_m61(b) % M != port.mod_m61(c):
            raise SystemExit(f"bench batched: product {i} failed the residue check")

    def one_by_one(_):
        for i in range(nprod):
            a_ptr, n_a, b_ptr, n_b, o_ptr = prods[i]
            bb.mul_device(a_ptr, n_a, b_ptr, n_b, o_ptr, stream=sp, method=bb.BGPU_METHOD_NTT)
    dout.zero_()
    one_by_one(0)
    bb.device_status(sp)
    if not np.array_equal(dout.cpu().numpy().view(np.uint64), host):
        raise SystemExit("bench batched: the batch differs from one plain NTT call per product")
    ms_single = _event_ms(torch, stream, one_by_one, 1)
    bb.device_status(sp)
    launches = plan.launches
    plan.close()
    # the same batch with every NTT class on its own launches (parallel graph
    # branches): the alternative form, timed and compared beside the default
    plan_pc = bb.BatchPlan(prods, flags=bb.BGPU_BATCH_PER_CLASS)
    dout.zero_()
    for _ in range(2):
        plan_pc.run(sp)
    bb.device_status(sp)
    ms_pc = _event_ms(torch, stream, lambda i: plan_pc.run(sp), runs)
    bb.device_status(sp)
    launches_pc = plan_pc.launches
    plan_pc.close()
    if not np.array_equal(dout.cpu().numpy().view(np.uint64), host):
        raise SystemExit("bench batched: the per-class launch sets differ from the default plan")
    verified = "residue mod 2^61-1 and identical to one plain NTT call, every product"
    from oracle.pyoracle import Reference, have_reference

    if have_reference() and ref_every:
        ref = Reference()
        ref.init_thread_pool(ref_pool_threads())
        for i in range(0, nprod, ref_every):
            a = big[offs_a[i]:offs_a[i] + na[i]]
            b = big[offs_b[i]:offs_b[i] + nb[i]]
            c = np.trim_zeros(host[offs_o[i]:offs_o[i] + outn[i]], "b")
            if not np.array_equal(c, ref.mul(a, b)):
                raise SystemExit(f"bench batched: product {i} differs from the reference's _mul")
        verified += f"; every {ref_every}th product limb-exact vs the reference's _mul"
    return {"products": nprod, "operand_bits": "log-uniform [2^10, 2^22]",
            "batched": {"ms_per_batch": ms_batch, "products_per_s": nprod / (ms_batch * 1e-3),
                        "launches_per_batch": launches, "graph_launches": 1,
                        "plan_build_s": t_plan},
            "per_class_launch_sets": {"ms_per_batch": ms_pc, "products_per_s": nprod / (ms_pc * 1e-3),
                                      "launches_per_batch": launches_pc, "speedup": ms_single / ms_pc,
                                      "note": "BGPU_BATCH_PER_CLASS: every NTT class its own four "
                                              "launches on parallel graph branches; same outputs"},
            "one_plain_ntt_launch_per_product": {"ms": ms_single,
                                                 "products_per_s": nprod / (ms_single * 1e-3),
                                                 "launches": 4 * nprod},
            "speedup": ms_single / ms_batch, "verified": verified}


def batched_same_size_form(bb, torch, device, port, A, B, count: int = 32, runs: int = 10):
    """The headline product batched: `count` independent 2^24 x 2^24-bit
    products in one batch plan (one NTT class, one graph launch), operands
    resident; per-product time and the fraction of the reference's two-pass
    HBM model it reaches."""
    count = min(count, A.shape[0])
    na, nb = A.shape[1], B.shape[1]
    dA = torch.from_numpy(np.ascontiguousarray(A[:count]).view(np.int64)).to(device)
    dB = torch.from_numpy(np.ascontiguousarray(B[:count]).view(np.int64)).to(device)
    dO = torch.empty((count, na + nb), dtype=torch.int64, device=device)
    plan = bb.BatchPlan([(dA[i].data_ptr(), na, dB[i].data_ptr(), nb, dO[i].data_ptr())
                         for i in range(count)])
    stream = torch.cuda.Stream(device)
    sp = stream.cuda_stream
    for _ in range(2):
        plan.run(sp)
    bb.device_status(sp)
    ms = _event_ms(torch, stream, lambda i: plan.run(sp), runs)
    bb.device_status(sp)
    launches = plan.launches
    plan.close()
    out = dO.cpu().numpy().view(np.uint64)
    M = (1 << 61) - 1
    for i in range(count):
        if port.mod_m61(A[i]) * port.mod_m61(B[i]) % M != port.mod_m61(out[i]):
            raise SystemExit(f"bench batched 2^24: product {i} failed the residue check")
    verified = "residue mod 2^61-1, every product"
    from oracle.pyoracle import Reference, have_reference

    if have_reference():
        ref = Reference()
        ref.init_thread_pool(ref_pool_threads())
        if not np.array_equal(out[count - 1], ref.mul(A[count - 1], B[count - 1])):
            raise SystemExit("bench batched 2^24: the last product differs from the reference's _mul")
        verified += "; the last product limb-exact vs the reference's _mul"
    per = ms / count
    model = reference_model_bytes(na, nb)
    return {"products": count, "ms_per_batch": ms, "us_per_product": per * 1e3,
            "products_per_s": 1e3 / per, "launches_per_batch": launches,
            "reference_model_frac": model / (per * 1e-3) / 1e9 / measured_peaks()[0],
            "verified": verified}


def tree_form(bb, torch, device, port, nleaves: int = 1 << 20, reps: int = 3, cpu: bool = True):
    """Config "product tree": 2^20 seeded u64 leaves in [2^32, 2^64) multiplied
    pairwise level by level (each level one set of launches) to one ~2^26-bit
    product; the reference BigInt tree timed on the host beside it."""
    rng = np.random.default_rng(SEED + 5)
    leaves = rng.integers(1 << 32, 2**64, nleaves, dtype=np.uint64, endpoint=False)
    width = 1 << max(0, (nleaves - 1).bit_length())
    dl = _dev_limbs(torch, device, leaves)
    dout = torch.empty(width, dtype=torch.int64, device=device)
    bb.product_tree_device(dl.data_ptr(), nleaves, dout.data_ptr(), width)
    times = []
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        bb.product_tree_device(dl.data_ptr(), nleaves, dout.data_ptr(), width)
        times.append(time.perf_counter() - t0)
    launches = bb.last_launch_count()
    got = dout.cpu().numpy().view(np.uint64)
    M = (1 << 61) - 1
    r = 1
    for x in leaves.tolist():
        r = r * (x % M) % M
    if port.mod_m61(got) != r:
        raise SystemExit("bench tree: residue check failed")
    res = {"leaves": nleaves, "levels": (nleaves - 1).bit_length(), "launches": launches,
           "ms": 1e3 * statistics.median(times), "products_per_s": (nleaves - 1) / statistics.median(times),
           "result_bits": int(np.count_nonzero(got) and (len(np.trim_zeros(got, "b")) * 64)),
           "verified": "residue mod 2^61-1 of the product of all leaves"}
    from oracle.pyoracle import Reference, have_reference

    if have_reference():
        ref = Reference()
        ref.init_thread_pool(ref_pool_threads())
        t0 = time.perf_counter()
        want = ref.product_tree_digits(leaves)
        t_ref = time.perf_counter() - t0
        if not np.array_equal(limbs_to_digits28_np(got), want):
            raise SystemExit("bench tree: the product differs from the reference's BigInt tree")
        res["verified"] += "; limb-exact vs the reference's BigInt tree"
        if cpu:
            res["cpu_reference"] = {"s": t_ref, "threads": ref_pool_threads(),
                                    "call": "BigInt::operator* pairwise tree"}
    return res


# ---- arms --------------------------------------------------------------------------

def run_reference_arm(args) -> None:
    """The reference's own CPU multiply (`_mul`, from oracle/_ref) on the host
    cores: K products after W warm-up products at each thread count of
    `cpu_thread_counts()`, each count in a process of its own; the line's
    value is the fastest count, and every count is listed."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    rows = cpu_reference_rates(args.bits, seconds=0.0, max_reps=args.steps, min_reps=args.steps,
                               warmup=args.warmup)
    best = max(rows, key=lambda r: r["rate"])
    value, cores, kind = best["rate"], best["threads"], best["kind"]
    line = {
        "impl": "reference",
        "metric": "bit-exact products/s (2^24 x 2^24-bit multiply)",
        "value": value, "unit": "products/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": workload_name(args.bits), "call": "bigint::mul::_mul",
                   "threads": cores, "parallelism": "host threads (init_thread_pool)",
                   "thread_counts": {str(r["threads"]): {"products_per_s": r["rate"], "reps": r["reps"]}
                                     for r in rows},
                   "physical_cores": physical_cores(), "logical_cpus": host_cores()},
        "cpu_baseline": {"value": value, "unit": "products/s", "cores": cores, "kind": kind,
                         "sample": f"{args.steps} products of the full workload after {args.warmup} "
                                   f"warm-up products, at {', '.join(str(r['threads']) for r in rows)} "
                                   f"threads (value: the fastest, {cores})"},
        "e2e": {"value": value, "unit": "products/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_gpu_arm(args) -> None:
    import torch

    world, rank, local = dist_env()
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import bigint_b200 as bb
    from oracle.pyoracle import Port

    bb.init(local)
    npairs = pairs_beyond_l2(args.bits)
    A, B = make_operands(args.bits, pairs=npairs)
    na = nb = A.shape[1]
    dA = torch.from_numpy(A.view(np.int64)).to(device)
    dB = torch.from_numpy(B.view(np.int64)).to(device)
    dOut = torch.empty((npairs, na + nb), dtype=torch.int64, device=device)
    stream = torch.cuda.Stream(device)
    sptr = stream.cuda_stream

    def step(i, flags=bb.BGPU_INDEPENDENT):
        # the products are independent: each one's transform may start under
        # the previous product's carry scan (BGPU_INDEPENDENT)
        k = i % npairs
        bb.mul_device(dA[k].data_ptr(), na, dB[k].data_ptr(), nb, dOut[k].data_ptr(), stream=sptr,
                      method=flags)

    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            step(i)
    bb.device_status(sptr)
    launches_per_step = bb.last_launch_count()

    # Timed region: windows of exactly K back-to-back products on one stream,
    # each bracketed by a barrier and a device synchronize on both sides and
    # timed with CUDA events on the launching stream.  Step i uses operand
    # pair i mod npairs; all pairs together exceed L2, so no step finds its
    # inputs cached by the previous one.  The window repeats until about
    # `--window-seconds` of device time (at least 5 windows) so the clock
    # sampler sees the whole run; the reported time is the median window.
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dOut.zero_()  # every output checked below comes from the timed products

    def window(flags, first_step):
        barrier(world, device)
        torch.cuda.synchronize(device)
        with torch.cuda.stream(stream):
            h0 = time.perf_counter()
            t0.record(stream)
            for i in range(args.steps):
                step(first_step + i, flags)
            t1.record(stream)
            issue_s = time.perf_counter() - h0
        torch.cuda.synchronize(device)
        barrier(world, device)
        return t0.elapsed_time(t1), issue_s

    first_ms, _ = window(bb.BGPU_INDEPENDENT, args.warmup)
    nwin = int(reduce_max(float(min(2000, max(5, round(args.window_seconds * 1e3 / max(first_ms, 1e-3))))),
                          world, device))
    win_ms, issue = [], []
    with ClockSampler(pci_bus_id(device)) as clk:
        for w in range(nwin):
            ms, iss = window(bb.BGPU_INDEPENDENT, args.warmup + w * args.steps)
            win_ms.append(ms)
            issue.append(iss)
    bb.device_status(sptr)
    total_ms = reduce_max(statistics.median(win_ms), world, device)
    clocks = clk.summary()
    out_timed = dOut.cpu().numpy().view(np.uint64)

    # The same K products without the flag: every product fully after the
    # previous one (what a caller gets without promising independence).
    seq_win = [window(0, args.warmup + w * args.steps)[0] for w in range(max(5, nwin // 4))]
    bb.device_status(sptr)
    seq_ms = reduce_max(statistics.median(seq_win), world, device)

    # Diagnostic of the host launches: the same K products enqueued behind a
    # bounded GPU sleep (torch.cuda._sleep, four times their host issue time),
    # so every launch is queued before the first product starts.  When the
    # timed windows' launches are hidden, both give the same time per product.
    sleep_cycles = int(min(2e9, 4 * max(issue) * 2.0e9))

    def prequeued_window(first_step):
        torch.cuda.synchronize(device)
        with torch.cuda.stream(stream):
            torch.cuda._sleep(sleep_cycles)
            t0.record(stream)
            for i in range(args.steps):
                step(first_step + i)
            t1.record(stream)
        torch.cuda.synchronize(device)
        return t0.elapsed_time(t1)

    preq_ms = None
    if hasattr(torch.cuda, "_sleep"):  # torch's own bounded GPU spin (a private helper)
        preq_win = [prequeued_window(args.warmup + w * args.steps) for w in range(5)]
        bb.device_status(sptr)
        preq_ms = reduce_max(statistics.median(preq_win), world, device)

    # Roofline pass: the same K products again with CUDA events recorded on
    # the launching stream between the kernels of every product (kept out of
    # the timed region above because an event between two kernels stops the
    # next launch from overlapping the previous kernel's tail).
    bb.set_kernel_timing(True)
    with torch.cuda.stream(stream):
        for i in range(args.steps):
            step(args.warmup + i)
    torch.cuda.synchronize(device)
    ktimes, kcount = bb.kernel_times()
    bb.set_kernel_timing(False)
    bb.device_status(sptr)

    # correctness of every output slot the timed windows wrote (the
    # overlapped pass) and of the last pass: residue identity mod 2^61-1, and
    # the two passes agree; one timed product limb-exact against the
    # reference's own _mul (oracle/_ref), outside every timed region
    port = Port()
    M = (1 << 61) - 1
    out_host = dOut.cpu().numpy().view(np.uint64)
    written = sorted({(args.warmup + i) % npairs for i in range(args.steps * nwin)})
    for k in written:
        if (port.mod_m61(A[k]) * port.mod_m61(B[k])) % M != port.mod_m61(out_timed[k]):
            raise SystemExit(f"bench: timed product {k} failed the mod 2^61-1 residue check")
        if not np.array_equal(out_timed[k], out_host[k]):
            raise SystemExit(f"bench: product {k} differs between the overlapped and the plain pass")
    verified = "residue mod 2^61-1, every output slot of the timed windows"
    from oracle.pyoracle import Reference, have_reference

    if have_reference() and rank == 0:
        k = written[0]
        ref = Reference()
        ref.init_thread_pool(ref_pool_threads())
        if not np.array_equal(out_timed[k], ref.mul(A[k], B[k])):
            raise SystemExit(f"bench: timed product {k} differs from the reference's _mul")
        verified += f"; product {k} limb-exact vs the reference's bigint::mul::_mul"

    # e2e through the public host API from pinned buffers: bgpu_mul_u64_many,
    # which pipelines a list of host-resident products (every product copies
    # its operands up and its product back; the copies of neighbouring
    # products overlap the multiplies), and the one-product synchronous call
    # (bgpu_mul_u64) beside it.
    pA = torch.from_numpy(A.view(np.int64)).pin_memory().numpy().view(np.uint64)
    pB = torch.from_numpy(B.view(np.int64)).pin_memory().numpy().view(np.uint64)
    pOut = torch.empty((npairs, na + nb), dtype=torch.int64).pin_memory().numpy().view(np.uint64)
    e2e_steps = min(args.steps, 400)  # the timed region's K products (the pipeline fills and drains once)
    pairs = [(pA[i % npairs], pB[i % npairs]) for i in range(e2e_steps)]
    outs = [pOut[i % npairs] for i in range(e2e_steps)]
    bb.mul_many(pairs[:4], outs[:4])  # warm-up
    e2e_win = []
    for _ in range(5):  # five windows of the K host-resident products; the median one
        torch.cuda.synchronize(device)
        barrier(world, device)
        te = time.perf_counter()
        bb.mul_many(pairs, outs)
        e2e_win.append(time.perf_counter() - te)
    e2e_s = reduce_max(statistics.median(e2e_win), world, device)
    for k in written:
        if k < e2e_steps and not np.array_equal(pOut[k], out_host[k]):
            raise SystemExit("bench: host-API product differs from the device-resident product")
    single_steps = min(e2e_steps, 20)
    for i in range(2):
        bb.mul(pA[i], pB[i], out=pOut[i])
    barrier(world, device)
    te = time.perf_counter()
    for i in range(single_steps):
        bb.mul(pA[i % npairs], pB[i % npairs], out=pOut[i % npairs])
    single_s = reduce_max(time.perf_counter() - te, world, device)

    # roofline of the dominant kernel
    log_n = (2 * na + 2 * nb - 2).bit_length()
    mean_k = dict(ktimes)
    dom = max(mean_k, key=mean_k.get)
    dom_bytes = kernel_bytes(dom, na, nb, log_n, square=False)
    peak, peak_kind = measured_peaks()
    achieved = dom_bytes / (mean_k[dom] * 1e-3) / 1e9
    prod_ms = total_ms / args.steps
    model_b = reference_model_bytes(na, nb)

    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank != 0:
        return

    forms = None
    if not args.no_forms:
        torch.cuda.synchronize(device)
        forms = {"plain_2p20": plain_2p20_form(bb, torch, device, port, cpu=not args.no_cpu_baseline),
                 "batched_2p24": batched_same_size_form(bb, torch, device, port, A, B),
                 "ntt_size_sweep": sweep_form(bb, torch, device, port),
                 "fp64_fft": fft_form(bb, torch, device),
                 "fast_pow": fast_pow_form(bb, port, cpu=not args.no_cpu_baseline),
                 "mul_digits_2p24": mul_digits_form(bb, port, cpu=not args.no_cpu_baseline),
                 "reciprocal_2p24": reciprocal_form(bb, cpu=not args.no_cpu_baseline),
                 "divmod_2p24": divmod_form(bb, port, cpu=not args.no_cpu_baseline),
                 "bigfloat_print_2p22": bigfloat_print_form(bb, cpu=not args.no_cpu_baseline),
                 "decimal_print_2p22": decimal_print_form(bb, cpu=not args.no_cpu_baseline),
                 "decimal_parse_5m": decimal_parse_form(bb, cpu=not args.no_cpu_baseline),
                 "batched_4096": batched_form(bb, torch, device, port),
                 "product_tree_2p20": tree_form(bb, torch, device, port,
                                                cpu=(rank == 0 and not args.no_cpu_baseline))}

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        rows = cpu_reference_rates(args.bits, args.cpu_seconds / len(cpu_thread_counts()), 50)
        best = max(rows, key=lambda r: r["rate"])
        cpu = {"value": best["rate"], "unit": "products/s", "cores": best["threads"], "kind": best["kind"],
               "sample": "; ".join(f"{r['threads']} threads: {r['reps']} full 2^24 x 2^24-bit products in "
                                   f"{r['seconds']:.1f} s ({r['rate']:.2f}/s)" for r in rows) +
                         f" ({'bigint::mul::_mul' if best['kind'] == 'reference' else 'C port ntt_mul'}; "
                         f"value: the fastest count)",
               "physical_cores": physical_cores(), "logical_cpus": host_cores()}

    value = world * args.steps / (total_ms * 1e-3)
    line = {
        "metric": "bit-exact products/s (2^24 x 2^24-bit multiply)",
        "value": value, "unit": "products/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": prod_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": workload_name(args.bits), "method": "ntt",
                   "transform_points": 1 << log_n, "digit_bits": 32,
                   "l2": f"inputs larger than L2: {npairs} distinct operand pairs "
                         f"({npairs * 2 * na * 8 >> 20} MiB) cycled, steps back to back",
                   "parallelism": f"replicas x{world}", "verified": verified,
                   "pipelining": "independent products (BGPU_INDEPENDENT): each product's forward "
                                 "transform starts under the previous product's carry scan",
                   "timing": f"median of {nwin} windows of exactly K={args.steps} products, each window "
                             "bracketed by barrier + synchronize, CUDA events on the launching stream; "
                             "max over ranks",
                   "windows_ms": {"median": statistics.median(win_ms), "min": min(win_ms),
                                  "max": max(win_ms), "count": nwin},
                   "host_issue_us_per_product": statistics.median(issue) / args.steps * 1e6,
                   "host_issue_note": "host time to enqueue one product (4 launches through the C-ABI); "
                                      "below the device time per product, the launches are hidden",
                   "prequeued_us_per_product": None if preq_ms is None else preq_ms / args.steps * 1e3,
                   "prequeued_note": "the same K products with every launch queued before the first one "
                                     "starts (behind a GPU sleep), median of 5 windows: equal to ms_per_step "
                                     "when the timed windows' host launches are hidden"},
        "sequential": {"ms_per_step": seq_ms / args.steps, "value": world * args.steps / (seq_ms * 1e-3),
                       "note": "the same products without BGPU_INDEPENDENT, each after the previous "
                               f"(median of {len(seq_win)} windows)"},
        "e2e": {"value": world * e2e_steps / e2e_s, "unit": "products/s",
                "h2d_bytes_per_step": (na + nb) * 8, "d2h_bytes_per_step": (na + nb) * 8,
                "api": f"bgpu_mul_u64_many over {e2e_steps} host-resident products (pinned), "
                       "median of 5 calls",
                "single_call": {"value": world * single_steps / single_s, "unit": "products/s",
                                "api": "bgpu_mul_u64, one synchronous call per product"}},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": profiled_traffic(dom), "algorithmic_bytes": dom_bytes,
                     "kernel_ms": mean_k[dom], "kernels_ms": mean_k, "kernel_samples": kcount,
                     "kernel_timing": "events between the kernels, second pass of the same K products",
                     "reference_model": {"bytes_per_product": model_b,
                                         "achieved": model_b / (prod_ms * 1e-3) / 1e9,
                                         "frac": model_b / (prod_ms * 1e-3) / 1e9 / peak},
                     "compute": compute_roofline(mean_k, dom, prod_ms, clocks.get("sm_mhz"),
                                                 source_mul_counts(na, nb, log_n, log_n - bb.get_split(log_n),
                                                                   bb.get_split(log_n), False))},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": launches_per_step * args.steps,
        "forms": forms,
    }
    print(json.dumps(line))


FORMS = ("plain_2p20", "batched_2p24", "ntt_size_sweep", "fp64_fft", "fast_pow", "mul_digits_2p24", "reciprocal_2p24",
         "divmod_2p24", "bigfloat_print_2p22", "decimal_print_2p22", "decimal_parse_5m", "batched_4096",
         "product_tree_2p20")


def run_profile_case(args) -> None:
    """A short, fixed run for profilers: `--profile-case K` products of the
    headline workload (device resident, BGPU_INDEPENDENT, one stream), then
    exit.  Prints only a status line; not a measurement."""
    import torch

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    import bigint_b200 as bb

    bb.init(0)
    npairs = pairs_beyond_l2(args.bits)
    A, B = make_operands(args.bits, pairs=npairs)
    na = nb = A.shape[1]
    dA = torch.from_numpy(A.view(np.int64)).to(device)
    dB = torch.from_numpy(B.view(np.int64)).to(device)
    dOut = torch.zeros((npairs, na + nb), dtype=torch.int64, device=device)
    stream = torch.cuda.Stream(device)
    with torch.cuda.stream(stream):
        for i in range(args.profile_case):
            k = i % npairs
            bb.mul_device(dA[k].data_ptr(), na, dB[k].data_ptr(), nb, dOut[k].data_ptr(),
                          stream=stream.cuda_stream, method=bb.BGPU_INDEPENDENT)
    bb.device_status(stream.cuda_stream)
    torch.cuda.synchronize(device)
    print(json.dumps({"profile_case": args.profile_case, "bits": args.bits, "status": "ok"}))


def run_single_form(args) -> None:
    """One of the other configurations alone (for profiling it): prints
    {"form": name, "result": ...}."""
    import torch

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    import bigint_b200 as bb
    from oracle.pyoracle import Port

    bb.init(0)
    port = Port()
    name = args.form
    if name == "plain_2p20":
        res = plain_2p20_form(bb, torch, device, port, cpu=not args.no_cpu_baseline)
    elif name == "batched_2p24":
        A, B = make_operands(args.bits, pairs=32)
        res = batched_same_size_form(bb, torch, device, port, A, B)
    elif name == "ntt_size_sweep":
        res = sweep_form(bb, torch, device, port)
    elif name == "fp64_fft":
        res = fft_form(bb, torch, device)
    elif name == "fast_pow":
        res = fast_pow_form(bb, port, cpu=not args.no_cpu_baseline)
    elif name == "mul_digits_2p24":
        res = mul_digits_form(bb, port, cpu=not args.no_cpu_baseline)
    elif name == "reciprocal_2p24":
        res = reciprocal_form(bb, cpu=not args.no_cpu_baseline)
    elif name == "divmod_2p24":
        res = divmod_form(bb, port, cpu=not args.no_cpu_baseline)
    elif name == "bigfloat_print_2p22":
        res = bigfloat_print_form(bb, cpu=not args.no_cpu_baseline)
    elif name == "decimal_print_2p22":
        res = decimal_print_form(bb, cpu=not args.no_cpu_baseline)
    elif name == "decimal_parse_5m":
        res = decimal_parse_form(bb, cpu=not args.no_cpu_baseline)
    elif name == "batched_4096":
        res = batched_form(bb, torch, device, port)
    else:
        res = tree_form(bb, torch, device, port, cpu=not args.no_cpu_baseline)
    print(json.dumps({"form": name, "result": res}))


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--bits", type=int, default=OPERAND_BITS)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--window-seconds", type=float, default=0.25,
                    help="device time the K-product window is repeated for (median window reported)")
    ap.add_argument("--profile-case", type=int, default=0,
                    help="run this many headline products and exit (for ncu; prints no measurement)")
    ap.add_argument("--cpu-worker", type=int, default=0, help=argparse.SUPPRESS)
    ap.add_argument("--cpu-max-reps", type=int, default=50, help=argparse.SUPPRESS)
    ap.add_argument("--cpu-min-reps", type=int, default=1, help=argparse.SUPPRESS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the other configurations (size sweep, FFT form, batch, tree)")
    ap.add_argument("--form", choices=FORMS, default=None,
                    help="run only this one of the other configurations and print its result")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.cpu_worker:
        run_cpu_worker(args)
        return
    if args.profile_case:
        run_profile_case(args)
        return
    if args.form:
        run_single_form(args)
        return
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_gpu_arm(args)


if __name__ == "__main__":
    main()
