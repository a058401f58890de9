"""Autotuner: measures on the current GPU the choices the engine makes per
product size and writes them as a tuning table (``bgpu_load_tuning`` format).

The reference hard-codes its dispatch (``_mul``, include/bigint/mul.h:208-220:
brute up to 16384 total bits, FFT up to ``fft::MAX_TOTAL_BITS``, NTT above)
and has one radix-2 transform schedule (src/mul/ntt_multithread.cpp:333-379).
Here each choice is timed on the device:

* transform split: for every transform length 2^L (L = 12..25) the column
  length 2^c (row length 2^(L-c)) with the shortest device time per product,
  and separately (L = 10..22) the one with the highest throughput for the
  NTT classes of batch plans and product-tree levels;
* schoolbook vs Karatsuba vs NTT for single products, and for products
  inside a batch plan (one CTA per schoolbook or Karatsuba product vs a
  batched NTT class);
* the FP64 complex-FFT form vs the NTT on the host API: AUTO uses the FFT
  form only in the limb range where it was faster (never, if it never was).

Every product timed here is device resident; times are CUDA-event means over
back-to-back launches on one stream.  Usage::

    python -m bigint_b200.autotune [--out PATH] [--quick]

The package applies ``tuning_b200.txt`` (next to this file) at ``init()``
unless the environment variable BIGINT_B200_TUNING names another table (or
is set to the empty string for the built-in choices).
"""
from __future__ import annotations

import argparse
import datetime
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_TABLE = os.path.join(HERE, "tuning_b200.txt")


def _event_ms(torch, stream, fn, reps: int, warm: int = 3) -> float:
    with torch.cuda.stream(stream):
        for i in range(warm):
            fn(i)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for i in range(reps):
            fn(i)
        e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _rand_dev(torch, dev, rng, shape):
    return torch.from_numpy(rng.integers(0, 2**63, shape, dtype=np.int64)).to(dev)


def valid_splits(log_n: int) -> list[int]:
    """Column-length exponents the engine accepts for 2^log_n points (rows of
    2^15 points exist for transforms above 2^23 points only)."""
    out = []
    for l2 in range(2, 12):
        l1 = log_n - l2
        if 3 <= l1 <= (15 if log_n > 23 else 14):
            out.append(l2)
    return out


def tune_splits(bb, torch, dev, stream, log_ns, reps_small=40, reps_large=10):
    """Best column-length exponent per transform length (non-square products;
    squares share the table)."""
    sp = stream.cuda_stream
    res = {}
    for ln in log_ns:
        cands = valid_splits(ln)
        if not cands:
            continue
        n = 1 << (ln - 2)  # na = nb = 2^(L-2) limbs -> 2^L points of 32-bit digits
        pairs = int(min(16, max(2, (256 << 20) // (16 * n))))
        rng = np.random.default_rng(ln)
        A = _rand_dev(torch, dev, rng, (pairs, n))
        B = _rand_dev(torch, dev, rng, (pairs, n))
        O = torch.empty((pairs, 2 * n), dtype=torch.int64, device=dev)

        def run(i):
            k = i % pairs
            bb.mul_device(A[k].data_ptr(), n, B[k].data_ptr(), n, O[k].data_ptr(), stream=sp,
                          method=bb.BGPU_METHOD_NTT)

        times = {}
        reps = reps_small if ln < 22 else reps_large
        for l2 in cands:
            bb.set_split(ln, l2)
            times[l2] = _event_ms(torch, stream, run, reps)
            bb.device_status(sp)
        bb.set_split(ln, 0)
        default = bb.get_split(ln)
        best = min(times, key=times.get)
        res[ln] = {"best": best, "default": default, "ms": times}
        print(f"split 2^{ln}: best column 2^{best} {times[best] * 1e3:.1f} us "
              f"(default 2^{default} {times.get(default, float('nan')) * 1e3:.1f} us)", flush=True)
        del A, B, O
    return res


def tune_batch_splits(bb, torch, dev, stream, log_ns):
    """Best column-length exponent per transform length for the NTT classes of
    batch plans: throughput of a batch large enough to fill the GPU."""
    sp = stream.cuda_stream
    res = {}
    for ln in log_ns:
        cands = valid_splits(ln)
        if not cands:
            continue
        n = 1 << (ln - 2)
        count = int(max(8, min(1024, (1 << 25) >> ln)))
        rng = np.random.default_rng(100 + ln)
        A = _rand_dev(torch, dev, rng, (count, n))
        B = _rand_dev(torch, dev, rng, (count, n))
        O = torch.empty((count, 2 * n), dtype=torch.int64, device=dev)
        prods = [(A[i].data_ptr(), n, B[i].data_ptr(), n, O[i].data_ptr()) for i in range(count)]
        times = {}
        for l2 in cands:
            bb.set_batch_split(ln, l2)
            plan = bb.BatchPlan(prods)
            times[l2] = _event_ms(torch, stream, lambda i: plan.run(sp), 5, warm=2)
            bb.device_status(sp)
            plan.close()
        bb.set_batch_split(ln, 0)
        default = bb.get_batch_split(ln)
        best = min(times, key=times.get)
        res[ln] = {"best": best, "default": default, "ms": times, "count": count}
        print(f"batch split 2^{ln} x{count}: best column 2^{best} {times[best] * 1e3:.1f} us "
              f"(default 2^{default} {times.get(default, float('nan')) * 1e3:.1f} us)", flush=True)
        del A, B, O
    return res


def _threshold(rows):
    """Largest total limb count up to which the first method won at every
    tested size (rows: [(total_limbs, ms_first, ms_second)] ascending)."""
    best = 0
    for total, t1, t2 in rows:
        if t1 <= t2:
            best = total
        else:
            break
    return best


def _small_thresholds(rows):
    """rows: [(total_limbs, t_schoolbook, t_karatsuba, t_ntt)] ascending, inf
    where a method cannot run.  Schoolbook up to the largest total where it
    beat both others at every size so far; Karatsuba from there up to the
    largest total where it beat the NTT."""
    sb = 0
    for total, t_sb, t_ka, t_nt in rows:
        if t_sb <= min(t_ka, t_nt):
            sb = total
        else:
            break
    ka = 0
    for total, t_sb, t_ka, t_nt in rows:
        if total <= sb:
            continue
        if t_ka <= t_nt:
            ka = total
        else:
            break
    return sb, ka


def tune_small(bb, torch, dev, stream, sizes):
    """Single products na = nb = s: schoolbook, Karatsuba and NTT."""
    sp = stream.cuda_stream
    rng = np.random.default_rng(7)
    rows = []
    inf = float("inf")
    for s in sizes:
        A = _rand_dev(torch, dev, rng, (s,))
        B = _rand_dev(torch, dev, rng, (s,))
        O = torch.empty(2 * s, dtype=torch.int64, device=dev)
        t = []
        for m, ok in ((bb.BGPU_METHOD_SCHOOLBOOK, 2 * s <= 256), (bb.BGPU_METHOD_KARATSUBA, s <= 256),
                      (bb.BGPU_METHOD_NTT, True)):
            if not ok:
                t.append(inf)
                continue
            t.append(_event_ms(torch, stream, lambda i, m=m: bb.mul_device(
                A.data_ptr(), s, B.data_ptr(), s, O.data_ptr(), stream=sp, method=m), 50))
            bb.device_status(sp)
        rows.append((2 * s, *t))
        print(f"single {s}x{s} limbs: schoolbook {t[0] * 1e3:.1f} us, karatsuba {t[1] * 1e3:.1f} us, "
              f"ntt {t[2] * 1e3:.1f} us", flush=True)
    return (*_small_thresholds(rows), rows)


def tune_batch_small(bb, torch, dev, stream, sizes, count=1024):
    """Batches of `count` products na = nb = s through a batch plan whose
    crossovers force each method in turn."""
    sp = stream.cuda_stream
    rng = np.random.default_rng(11)
    rows = []
    inf = float("inf")
    keys = (bb.BGPU_TUNE_BATCH_SCHOOLBOOK_MAX_LIMBS, bb.BGPU_TUNE_BATCH_KARATSUBA_MAX_LIMBS)
    saved = [bb.get_tuning(k) for k in keys]
    for s in sizes:
        A = _rand_dev(torch, dev, rng, (count, s))
        B = _rand_dev(torch, dev, rng, (count, s))
        O = torch.empty((count, 2 * s), dtype=torch.int64, device=dev)
        prods = [(A[i].data_ptr(), s, B[i].data_ptr(), s, O[i].data_ptr()) for i in range(count)]
        t = []
        for sb_lim, ka_lim, ok in ((2 * s, 0, 2 * s <= 256), (0, 2 * s, s <= 256), (0, 0, True)):
            if not ok:
                t.append(inf)
                continue
            bb.set_tuning(keys[0], sb_lim)
            bb.set_tuning(keys[1], ka_lim)
            plan = bb.BatchPlan(prods)
            t.append(_event_ms(torch, stream, lambda i: plan.run(sp), 10))
            bb.device_status(sp)
            plan.close()
        rows.append((2 * s, *t))
        print(f"batch {count} x ({s}x{s}) limbs: schoolbook {t[0] * 1e3:.1f} us, "
              f"karatsuba {t[1] * 1e3:.1f} us, ntt {t[2] * 1e3:.1f} us", flush=True)
        del A, B, O
    for k, v in zip(keys, saved):
        bb.set_tuning(k, v)
    return (*_small_thresholds(rows), rows)


def tune_fft(bb, log_limbs):
    """Host API: device time of the FFT form (worst-case bound) vs the NTT,
    na = nb = 2^k limbs; returns the contiguous winning range or (0, 0)."""
    rng = np.random.default_rng(13)
    rows = []
    for k in log_limbs:
        n = 1 << k
        a = rng.integers(0, 2**64, n, dtype=np.uint64, endpoint=False)
        b = rng.integers(0, 2**64, n, dtype=np.uint64, endpoint=False)
        tf, tn = [], []
        for _ in range(4):
            _, sf = bb.fft_mul(a, b, stats=True)
            _, sn = bb.ntt_mul(a, b, stats=True)
            tf.append(sf.device_ms if not sf.fell_back else float("inf"))
            tn.append(sn.device_ms)
        rows.append((2 * n, min(tf[1:]), min(tn[1:])))
        print(f"fft vs ntt {n}x{n} limbs: fft {rows[-1][1] * 1e3:.1f} us, ntt {rows[-1][2] * 1e3:.1f} us",
              flush=True)
    wins = [r[0] for r in rows if r[1] < r[2]]
    if not wins:
        return (0, 0), rows
    return (min(wins), max(wins)), rows


def write_table(path: str, device: str, splits, bsplits, small, bsmall, fft, fft_rows) -> None:
    sb, ka, sb_rows = small
    bsb, bka, bsb_rows = bsmall
    lines = [f"# bigint_b200 tuning table for {device}",
             f"# written by bigint_b200/autotune.py at {datetime.datetime.now(datetime.timezone.utc).isoformat(timespec='seconds')}",
             "# split <log2 points> <log2 column length>   (device us per product: best / built-in)"]
    for ln in sorted(splits):
        r = splits[ln]
        lines.append(f"split {ln} {r['best']}    # {r['ms'][r['best']] * 1e3:.1f} / "
                     f"{r['ms'].get(r['default'], float('nan')) * 1e3:.1f}")
    lines.append("# batch_split <log2 points> <log2 column length>   (us per batch of `count` products:"
                 " best / built-in)")
    for ln in sorted(bsplits):
        r = bsplits[ln]
        lines.append(f"batch_split {ln} {r['best']}    # x{r['count']}: {r['ms'][r['best']] * 1e3:.1f} / "
                     f"{r['ms'].get(r['default'], float('nan')) * 1e3:.1f}")
    lines.append("# single products: schoolbook / Karatsuba / NTT (us), na + nb limbs")
    lines += [f"#   {t}: {a * 1e3:.1f} / {b * 1e3:.1f} / {c * 1e3:.1f}" for t, a, b, c in sb_rows]
    lines.append(f"schoolbook_max_limbs {sb}")
    lines.append(f"karatsuba_max_limbs {ka}")
    lines.append("# batches of 1024 products: schoolbook / Karatsuba / NTT class (us per batch)")
    lines += [f"#   {t}: {a * 1e3:.1f} / {b * 1e3:.1f} / {c * 1e3:.1f}" for t, a, b, c in bsb_rows]
    lines.append(f"batch_schoolbook_max_limbs {bsb}")
    lines.append(f"batch_karatsuba_max_limbs {bka}")
    lines.append("# FP64 FFT form vs NTT on the host API (device us), na + nb limbs")
    lines += [f"#   {t}: {a * 1e3:.1f} vs {b * 1e3:.1f}" for t, a, b in fft_rows]
    lines.append(f"fft_min_limbs {fft[0]}")
    lines.append(f"fft_max_limbs {fft[1]}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--quick", action="store_true", help="fewer transform lengths and sizes")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)

    import torch

    os.environ["BIGINT_B200_TUNING"] = ""  # measure from the built-in choices
    import bigint_b200 as bb

    bb.init(args.device)
    dev = torch.device("cuda", args.device)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    log_ns = range(12, 26, 3 if args.quick else 1)
    splits = tune_splits(bb, torch, dev, stream, log_ns)
    for ln, r in splits.items():  # later stages measure with the tuned splits
        bb.set_split(ln, r["best"])
    bsplits = tune_batch_splits(bb, torch, dev, stream, range(10, 23, 3 if args.quick else 1))
    for ln, r in bsplits.items():
        bb.set_batch_split(ln, r["best"])
    sizes = [8, 16, 32, 48, 64, 96, 128, 192, 256, 384] if not args.quick else [16, 64, 128, 256]
    small = tune_small(bb, torch, dev, stream, sizes)
    bsmall = tune_batch_small(bb, torch, dev, stream, sizes)
    fft, fft_rows = tune_fft(bb, range(8, 19, 2) if not args.quick else (10, 14))
    name = torch.cuda.get_device_name(dev)
    write_table(args.out, name, splits, bsplits, small, bsmall, fft, fft_rows)
    print(f"wrote {args.out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
