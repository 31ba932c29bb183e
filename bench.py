#!/usr/bin/env python
"""Benchmark: GKeys/s of the B200 LSD radix sort against its HBM roofline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload u32_full] [--no-breakdown]

A step is one full sort (upfront scan and histogram, every live onesweep
pass, finishing kernels) of 2^28 keys already resident in HBM (1 GiB, far
above the 126 MB L2); each step sorts its own unsorted copy. `value` is keys
sorted per second over the K timed steps (CUDA events on the sort's stream,
max over ranks). `e2e` times the host-slice C ABI call ts_sort_u32 on pinned
host memory: the copy in, the sort and the copy out, which the library
overlaps (chunked copies in, chunk sorts and device merges, sliced copies
out); the same call with the copies serialised is reported beside it. `roofline` is the
onesweep pass kernel: algorithmic bytes of one pass (read + write of every
key) over its CUDA-event duration, against the measured HBM copy bandwidth.
Under torchrun each rank sorts its own array (replicas: the crate's sort has
no cross-device step).

--impl reference times the crate's own algorithm on the host cores instead
(its C restatement, sort_parallel on every core), on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "GKeys/s on 1 B200 vs HBM roofline, bit-exact; learned/batched vs plain radix"

# name -> (key type, distribution, log2 n)
WORKLOADS = {
    "u32_full": ("u32", 0, 28), "u32_low_entropy": ("u32", 1, 28), "u32_range16": ("u32", 2, 28),
    "i32_full": ("i32", 0, 28), "i32_low_entropy": ("i32", 1, 28), "i32_range16": ("i32", 2, 28),
    "f32_full": ("f32", 0, 28), "f32_low_entropy": ("f32", 1, 28), "f32_range16": ("f32", 2, 28),
    "u64_full": ("u64", 0, 27), "u64_low_entropy": ("u64", 1, 27), "u64_range16": ("u64", 2, 27),
    "c1_u32_2p20": ("u32", 0, 20),
}
DIST_NAMES = ("full-entropy", "AND of 3 words", "16-bit range in the low bits")
NP = {"u32": np.uint32, "i32": np.int32, "f32": np.float32, "u64": np.uint64}
WIDTH = {"u32": 4, "i32": 4, "f32": 4, "u64": 8}


def radix_keys_np(a: np.ndarray) -> np.ndarray:
    """to_radix_key (src/key.rs:135-197) with numpy, for output checks."""
    if a.dtype == np.float32:
        b = a.view(np.uint32)
        return b ^ ((b.view(np.int32) >> 31).view(np.uint32) | np.uint32(0x80000000))
    if a.dtype == np.float64:
        b = a.view(np.uint64)
        return b ^ ((b.view(np.int64) >> 63).view(np.uint64) | np.uint64(1 << 63))
    if a.dtype == np.int32:
        return a.view(np.uint32) ^ np.uint32(0x80000000)
    if a.dtype == np.int64:
        return a.view(np.uint64) ^ np.uint64(1 << 63)
    return a


def expected_radix(host: np.ndarray) -> np.ndarray:
    """What the sort must return, as radix keys: numpy's sort of the input's
    radix keys. The sort by to_radix_key is the crate's definition of the
    output (tests/correctness.rs:6-8) and is unique for these types."""
    return np.sort(radix_keys_np(host))


def check_exact(out: np.ndarray, want_radix: np.ndarray) -> bool:
    """Byte-equal to the expected output (the radix transform is a bijection)."""
    return radix_keys_np(out).tobytes() == want_radix.tobytes()


def live_passes(keys: np.ndarray, width: int) -> int:
    """Digits (8-bit) that some key does not share with the others."""
    k = radix_keys_np(keys)
    diff = np.bitwise_or.reduce(k ^ k[0])
    live = 0
    for d in range(width):
        if (int(diff) >> (8 * d)) & 0xFF:
            col = (k >> k.dtype.type(8 * d)) & k.dtype.type(0xFF)
            live += int(np.any(col != col[0]))
    return live


def gen(kind: str, dist: int, n: int, seed: int) -> np.ndarray:
    from turbosort_b200 import workloads as W

    return W.scale(kind, dist, n, seed=seed)


class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1].split()[0]))
                    mx.append(float(f[2].split()[0]))
                except ValueError:
                    continue
                for name, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(name)
            os.unlink(self.path)
        except Exception:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_gbs() -> tuple[float, str]:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(name: str):
    """dram bytes per launch from a committed ncu summary, if one exists."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_sample_rate(kind: str, dist: int, n_full: int, budget_s: float, threads: int, seed: int,
                    serial: bool = False):
    """The oracle's sort_parallel, or with `serial` its sort on one core (the
    crate's algorithm restated in C), on a bounded sample of the workload:
    returns (GKeys/s, sample description)."""
    from oracle import oracle as O

    n = min(n_full, 1 << 24)
    base = gen(kind, dist, n, seed)
    work = base.copy()

    def run(a):
        if serial:
            O.sort_inplace(a)
        else:
            O.sort_parallel_inplace(a, threads)

    run(work)  # warm-up
    reps, total = 0, 0.0
    while total < budget_s and reps < 50:
        np.copyto(work, base)
        t0 = time.perf_counter()
        run(work)
        total += time.perf_counter() - t0
        reps += 1
    return n * reps / total / 1e9, f"{reps} sorts of 2^{n.bit_length() - 1} keys of the same distribution"


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O

    kind, dist, lg = WORKLOADS[args.workload]
    n_full = 1 << lg
    threads = os.cpu_count() or 1
    # size the sample so that warm-up + steps stay within ~2 minutes
    probe_n = min(n_full, 1 << 22)
    probe = gen(kind, dist, probe_n, 7)
    t0 = time.perf_counter()
    O.sort_parallel_inplace(probe, threads)
    per_key = (time.perf_counter() - t0) / probe_n
    n = n_full
    while n > (1 << 20) and per_key * n * (args.steps + args.warmup) > 120.0:
        n //= 2
    base = gen(kind, dist, n, 0x9E3779B97F4A7C15)
    work = base.copy()
    for _ in range(args.warmup):
        np.copyto(work, base)
        O.sort_parallel_inplace(work, threads)
    times = []
    for _ in range(args.steps):
        np.copyto(work, base)
        t0 = time.perf_counter()
        O.sort_parallel_inplace(work, threads)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = n * args.steps / total / 1e9
    sample = f"{args.steps} sorts of 2^{n.bit_length() - 1} of the workload's keys (full workload 2^{lg})"
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "GKeys/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * total / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": kind,
        "data": "synthetic (seeded xorshift64)",
        "config": workload_config(args.workload),
        "cpu_baseline": {"value": round(value, 4), "unit": "GKeys/s", "cores": threads, "kind": "port",
                         "sample": sample,
                         "what": "turbosort sort_parallel (src/parallel.rs) restated in C, pthreads on every core"},
        "e2e": {"value": round(value, 4), "unit": "GKeys/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(name: str, lg: int | None = None) -> dict:
    kind, dist, lg0 = WORKLOADS[name]
    lg = lg or lg0
    return {"workload": f"plain LSD sort of 2^{lg} {kind} keys, {DIST_NAMES[dist]} (seeded xorshift64), 8-bit digits",
            "name": name, "n": 1 << lg, "key_type": kind,
            "l2": "inputs larger than L2 (1 GiB vs 126 MB); each step sorts its own unsorted copy",
            "parallelism": "replicas"}


PIPE_CHUNKS = 8            # the library's default transfer pipeline
PIPE_MIN_BYTES = 64 << 20


def reduce_over_ranks(torch, dist_mod, ms: float, ok: bool, device: str) -> tuple[float, bool]:
    """The job's time is the slowest rank's (replicas start together after a
    barrier); the job is correct only if every rank's output checked out.
    Without a process group this rank is the job."""
    if dist_mod is None:
        return ms, ok
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist_mod.all_reduce(t, op=dist_mod.ReduceOp.MAX)
    okt = torch.tensor([0 if ok else 1], dtype=torch.int32, device=device)
    dist_mod.all_reduce(okt, op=dist_mod.ReduceOp.MAX)
    return float(t.item()), int(okt.item()) == 0


def whole_job_gkeys(world: int, n_per_rank: int, ms_per_step: float) -> float:
    """Keys sorted by all ranks per second (each rank sorts its own n keys a step)."""
    return world * n_per_rank / (ms_per_step / 1e3) / 1e9


def bench_device(ts, torch, ctx, kind, dist, lg, steps, warmup, seed, dist_mod, rank, world, timing=True):
    n = 1 << lg
    w = WIDTH[kind]
    host = gen(kind, dist, n, seed)
    live = live_passes(host, w)
    tdt = {"u32": torch.int32, "i32": torch.int32, "f32": torch.int32, "u64": torch.int64}[kind]
    master = torch.from_numpy(host.view(np.int64 if w == 8 else np.int32)).to(f"cuda:{ctx.device}")
    view_dt = {"u32": torch.uint32, "i32": torch.int32, "f32": torch.float32, "u64": torch.uint64}[kind]
    copies = [master.clone() for _ in range(steps + warmup)]
    del master
    for i in range(warmup):
        ts.sort(copies[i].view(view_dt), ctx)
    torch.cuda.synchronize()
    lib = ts.lib()
    if dist_mod is not None:
        dist_mod.barrier()
    torch.cuda.synchronize()
    ctx.reset_timings()
    ctx.enable_timing(timing)
    launches0 = lib.ts_ctx_launches(ctx.handle)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(steps):
        ts.sort(copies[warmup + i].view(view_dt), ctx)
    e1.record()
    torch.cuda.synchronize()
    if dist_mod is not None:
        dist_mod.barrier()
    ms = e0.elapsed_time(e1)
    launches = lib.ts_ctx_launches(ctx.handle) - launches0
    tm = ctx.timings()
    ctx.enable_timing(False)
    ctx.synchronize()
    info = ctx.last_sort_info()
    if info["tier"] == 3 and info["mode"] == 0:
        live = info["passes"]  # the scatter passes that ran (diverting may leave out low digits)
    out = copies[-1].cpu().numpy().view(NP[kind])
    del copies
    ok = check_exact(out, expected_radix(host))
    torch.cuda.empty_cache()
    return {"ms_total": ms, "launches": launches, "timings": tm, "ok": ok, "live": live, "n": n, "w": w,
            "divert_shift": info.get("divert_shift", 0)}


def sort_bytes_of(r: dict) -> int:
    """Algorithmic bytes of one sort: one upfront read, a read and a write per
    scatter pass, and one read of the keys to find the runs when it diverted."""
    nw = r["n"] * r["w"]
    return nw * (2 * r["live"] + 1) + (nw if r.get("divert_shift") else 0)


def bench_small(ts, torch, ctx, kind, dist, lg, steps, warmup, seed):
    """Config 1 (2^20 keys): a latency-bound sort. One device buffer is
    refilled from a master copy before each step (outside the events) and
    sorted in place, so repeated calls replay the library's captured launch
    sequence (CUDA graph); CUDA events bracket each sort alone."""
    n = 1 << lg
    host = gen(kind, dist, n, seed)
    w = WIDTH[kind]
    view_dt = {"u32": torch.uint32, "i32": torch.int32, "f32": torch.float32, "u64": torch.uint64}[kind]
    master = torch.from_numpy(host.view(np.int64 if w == 8 else np.int32)).to(f"cuda:{ctx.device}")
    d = torch.empty_like(master)
    times = []
    for i in range(warmup + steps):
        d.copy_(master)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        ts.sort(d.view(view_dt), ctx)
        e1.record()
        torch.cuda.synchronize()
        if i >= warmup:
            times.append(e0.elapsed_time(e1))
    ok = check_exact(d.cpu().numpy().view(NP[kind]), expected_radix(host))
    ms = statistics.median(times)
    return {"gkeys_s": round(n / (ms / 1e3) / 1e9, 2), "ms": round(ms, 4), "ok": ok,
            "what": "median of per-sort CUDA-event times, same buffer each step (graph replay)"}


def bench_by_key(ts, torch, ctx, lg, steps, warmup, peak):
    """Config 3: stable sort_by_key_with_buffer of 2^lg records keyed by u64
    Zipf(1.1) keys over 2^20 distinct values; the records are 16 bytes
    {u64 id = original index, u32 a, u32 b}; then apply_order on a second
    u32 slice. A step = order() + moving both slices, all on the device."""
    from turbosort_b200 import workloads as W

    n = 1 << lg
    keys = W.zipf_u64(n)
    dev = f"cuda:{ctx.device}"
    dk = torch.from_numpy(keys.view(np.int64)).to(dev)
    g = torch.Generator(device=dev)
    g.manual_seed(3)
    rec = torch.empty((n, 4), dtype=torch.int32, device=dev)
    ids = torch.arange(n, dtype=torch.int64, device=dev)
    rec[:, 0:2] = ids.view(torch.int32).view(n, 2)
    rec[:, 2:4] = torch.randint(-2**31, 2**31 - 1, (n, 2), dtype=torch.int32, device=dev, generator=g)
    side = torch.randint(-2**31, 2**31 - 1, (n,), dtype=torch.int32, device=dev, generator=g)
    side0 = side.clone()
    order = torch.empty(n, dtype=torch.int32, device=dev)
    lib = ts.lib()

    def step():
        ctx._check(lib.ts_sort_keys_order_dev_u64(ctx.handle, dk.data_ptr(), n, order.data_ptr()))
        ctx._check(lib.ts_apply_order_dev(ctx.handle, rec.data_ptr(), n, 16, order.data_ptr(), n))
        ctx._check(lib.ts_apply_order_dev(ctx.handle, side.data_ptr(), n, 4, order.data_ptr(), n))

    step()  # checked below: records and side slice moved once
    ctx.synchronize()
    torch.cuda.synchronize()
    o = order.to(torch.int64)
    kk = dk[o].cpu().numpy().view(np.uint64)
    oo = o.cpu().numpy()
    sorted_ok = bool(np.all(kk[1:] >= kk[:-1]))
    eq = kk[1:] == kk[:-1]
    stable_ok = bool(np.all(oo[1:][eq] > oo[:-1][eq]))
    perm_ok = bool(np.array_equal(np.sort(oo), np.arange(n)))
    rec_ok = bool(torch.equal(rec[:, 0:2].contiguous().view(torch.int64).view(-1), o))
    side_ok = bool(torch.equal(side, side0[o]))
    ok = sorted_ok and stable_ok and perm_ok and rec_ok and side_ok
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    ctx.reset_timings()
    ctx.enable_timing(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ctx.enable_timing(False)
    tm = ctx.timings()
    ms = e0.elapsed_time(e1) / steps
    sweep_ms = tm.get("onesweep", (0.0, 0))[0] / steps
    gather_ms = tm.get("gather", (0.0, 0))[0] / steps
    del rec, side, side0, dk, order
    torch.cuda.empty_cache()
    return {"gkeys_s": round(n / (ms / 1e3) / 1e9, 3), "ms": round(ms, 3), "order_ms": round(ms - gather_ms, 3),
            "apply_order_ms": round(gather_ms, 3), "onesweep_ms": round(sweep_ms, 3),
            "what": "order() of 2^27 Zipf u64 keys + apply_order of 16-byte records and a u32 slice",
            "ok": ok, "checks": "sorted, stable (equal keys keep input order), permutation, records and side slice moved"}


def bench_tiny(ts, torch, ctx, steps):
    """Latency of one plain device sort of a short slice (the crate's tiny
    and small tiers, src/tiny.rs, src/small.rs): median CUDA-event time of a
    single call, same buffer each time."""
    out = {}
    for n in (17, 100, 256, 1000, 4096):
        host = np.random.default_rng(n).integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
        master = torch.from_numpy(host.view(np.int32)).to(f"cuda:{ctx.device}")
        d = torch.empty_like(master)
        times = []
        for i in range(steps + 3):
            d.copy_(master)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            ts.sort(d.view(torch.uint32), ctx)
            e1.record()
            torch.cuda.synchronize()
            if i >= 3:
                times.append(e0.elapsed_time(e1))
        ok = check_exact(d.cpu().numpy().view(np.uint32), expected_radix(host))
        out[str(n)] = {"us": round(1000 * statistics.median(times), 2), "ok": ok}
    return out


def bench_segments(ts, torch, ctx, kind, steps, warmup, per_segment=True, count=100_000, tune=True):
    """Config 4: 100,000 segments with lengths log-uniform on [1, 65536], keys
    of random bits, sorted in one segmented launch (graph replay, autotuned
    on-chip methods), against one plain sort call per segment."""
    from turbosort_b200 import workloads as W

    lengths = W.segment_lengths(count)
    offs = np.zeros(lengths.size + 1, dtype=np.uint64)
    offs[1:] = np.cumsum(lengths)
    n = int(offs[-1])
    bits = W.plain_u32(n, seed=0x2545F4914F6CDD1D)
    host = bits.view(np.float32) if kind == "f32" else bits
    dev = f"cuda:{ctx.device}"
    methods = ts.segments_autotune(4, ctx) if tune else ts.segments_methods(4, ctx)
    master = torch.from_numpy(bits.view(np.int32)).to(dev)
    d = torch.empty_like(master)
    d_off = torch.from_numpy(offs.view(np.int64)).to(dev)
    tdt = torch.float32 if kind == "f32" else torch.uint32
    for _ in range(warmup):
        d.copy_(master)
        ts.sort_segments(d.view(tdt), d_off, ctx)
    torch.cuda.synchronize()
    tot = 0.0
    for _ in range(steps):
        d.copy_(master)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        ts.sort_segments(d.view(tdt), d_off, ctx)
        e1.record()
        torch.cuda.synchronize()
        tot += e0.elapsed_time(e1)
    ms = tot / steps
    out = d.cpu().numpy().view(host.dtype)
    # every segment byte-equal to numpy's sort of its radix keys: one sort of
    # (segment index, radix key) pairs packed in 64 bits sorts all segments
    seg_id = np.repeat(np.arange(lengths.size, dtype=np.uint64), lengths.astype(np.int64))
    packed = (seg_id << np.uint64(32)) | radix_keys_np(host).astype(np.uint64)
    del seg_id
    packed.sort()
    want = (packed & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    del packed
    ok = check_exact(out, want)
    res = {"gkeys_s": round(n / (ms / 1e3) / 1e9, 3), "ms": round(ms, 3), "keys": n, "segments": int(lengths.size),
           "methods_names": ["bitonic", "radix-4", "radix-8", "msd", "warp"],
           "methods_per_bin": methods, "ok": ok,
           "roofline_frac": round(2 * n * 4 / (ms / 1e3) / 1e9 / measured_peak_gbs()[0], 3)}
    if per_segment:
        # the crate's way: one sort call per slice (here the plain device sort per segment)
        lib = ts.lib()
        f = getattr(lib, f"ts_sort_dev_{kind}")
        base = d.data_ptr()
        d.copy_(master)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        h = ctx.handle
        for s in range(lengths.size):
            lo = int(offs[s])
            f(h, base + 4 * lo, int(lengths[s]))
        e1.record()
        torch.cuda.synchronize()
        ps_ms = max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3)
        out2 = d.cpu().numpy().view(host.dtype)
        res["per_segment_ms"] = round(ps_ms, 1)
        res["speedup_vs_per_segment"] = round(ps_ms / ms, 1)
        res["ok"] = res["ok"] and out2.tobytes() == out.tobytes()
    del master, d, d_off
    torch.cuda.empty_cache()
    return res


def bench_learned(ts, torch, ctx, kind, steps, warmup, peak, lg=28, buckets_log2=14):
    """Config 5: the learned-partition sort against the plain device LSD on the
    same 2^lg keys: f64 lognormal(0, 2), u64 from 8 Gaussians (means in
    [0, 2^60], sigma 2^40), f32 uniform [0, 1) with 10% duplicates. Model: 1024
    leaves, 1% sample, 2^14 buckets, fallback at 4x the mean bucket. Both
    outputs must be identical bit for bit."""
    from turbosort_b200 import workloads as W

    n = 1 << lg
    host = {"lognormal_f64": W.lognormal_f64, "gauss_mix_u64": W.gauss_mix_u64,
            "unit_f32_dups": W.unit_f32_dups}[kind](n)
    w = host.itemsize
    dev = f"cuda:{ctx.device}"
    tdt = {"lognormal_f64": torch.float64, "gauss_mix_u64": torch.uint64, "unit_f32_dups": torch.float32}[kind]
    master = torch.from_numpy(host.view(np.int64 if w == 8 else np.int32)).to(dev)
    d = torch.empty_like(master)
    # the partition itself (the cost route off), against the plain sort with
    # and without diverting
    p = ts.learned_params(buckets_log2=buckets_log2, route_passes=0)

    def timed(fn):
        tot = 0.0
        for i in range(warmup + steps):
            d.copy_(master)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            r = fn()
            e1.record()
            torch.cuda.synchronize()
            if i >= warmup:
                tot += e0.elapsed_time(e1)
        return tot / steps, r

    ms_plain, _ = timed(lambda: ts.sort(d.view(tdt), ctx))
    plain_info = ctx.last_sort_info()
    plain_out = d.clone()
    ctx.set_divert(False)
    ms_plain_all, _ = timed(lambda: ts.sort(d.view(tdt), ctx))
    all_info = ctx.last_sort_info()
    ctx.set_divert(True)
    ok_all = bool(torch.equal(d, plain_out))
    d.copy_(master)
    st_default = ts.sort_learned(d.view(tdt), ts.learned_params(buckets_log2=buckets_log2), ctx)
    ms_learned, st = timed(lambda: ts.sort_learned(d.view(tdt), p, ctx))
    ok = bool(torch.equal(d, plain_out)) and ok_all
    # both byte-equal to numpy's sort of the input's radix keys
    ok &= check_exact(plain_out.cpu().numpy().view(host.dtype), expected_radix(host))
    del host
    launches0 = ts.lib().ts_ctx_launches(ctx.handle)
    d.copy_(master)
    ts.sort_learned(d.view(tdt), p, ctx)
    launches = ts.lib().ts_ctx_launches(ctx.handle) - launches0
    del master, d, plain_out
    torch.cuda.empty_cache()
    learned_bytes = n * w * 5  # predict read + partition read/write + bucket sort read/write
    return {"gkeys_s": round(n / (ms_learned / 1e3) / 1e9, 3), "ms": round(ms_learned, 3),
            "plain_gkeys_s": round(n / (ms_plain / 1e3) / 1e9, 3), "plain_ms": round(ms_plain, 3),
            "speedup_vs_plain": round(ms_plain / ms_learned, 3),
            "plain_passes": plain_info["passes"], "plain_divert_shift": plain_info["divert_shift"],
            "plain_all_passes_ms": round(ms_plain_all, 3), "plain_all_passes": all_info["passes"],
            "speedup_vs_plain_all_passes": round(ms_plain_all / ms_learned, 3),
            "default_route": {"routed_to_plain": int(st_default["reason"] == 4),
                              "est_plain_passes": st_default["est_plain_passes"]},
            "roofline_frac": round(learned_bytes / (ms_learned / 1e3) / 1e9 / peak, 3),
            "fell_back": st["fell_back"], "reason": st["reason"], "imbalance": round(st["imbalance"], 3),
            "max_bucket": st["max_bucket"], "max_cdf_error": round(st["max_cdf_error"], 5),
            "train_loss": [st["train_loss_first"], st["train_loss_last"]],
            "phase_ms": {k2: round(st[k2], 3) for k2 in ("ms_sample", "ms_train", "ms_partition", "ms_buckets")},
            "launches": int(launches), "keys": n, "ok": ok,
            "checks": "learned output == plain device sort output (with and without diverting) == numpy's sort "
                      "of the radix keys (bytes)"}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="u32_full", choices=sorted(WORKLOADS))
    ap.add_argument("--no-breakdown", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--log2n", type=int, default=None, help="override the workload's size (profiling runs)")
    ap.add_argument("--learned", default=None, choices=["lognormal_f64", "gauss_mix_u64", "unit_f32_dups"],
                    help="only the learned-partition comparison on this input (2^log2n keys, default 2^28)")
    ap.add_argument("--buckets-log2", type=int, default=14, help="buckets of the learned partition (with --learned)")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the tile autotuner (the library's measured defaults; for profiling runs)")
    ap.add_argument("--segments", default=None, choices=["u32", "f32"],
                    help="only the segmented-sort comparison (config 4) for these keys")
    ap.add_argument("--segment-count", type=int, default=100_000, help="segments (with --segments)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        run_reference(args)
        return
    if args.learned:
        import torch

        import turbosort_b200 as ts

        ctx = ts.Context(0)
        ctx.set_stream(torch.cuda.current_stream().cuda_stream)
        res = bench_learned(ts, torch, ctx, args.learned, args.steps, args.warmup, measured_peak_gbs()[0],
                            lg=args.log2n or 28, buckets_log2=args.buckets_log2)
        print(json.dumps({"learned": args.learned, **res}), flush=True)
        return

    if args.segments:
        import torch

        import turbosort_b200 as ts

        ctx = ts.Context(0)
        ctx.set_stream(torch.cuda.current_stream().cuda_stream)
        res = bench_segments(ts, torch, ctx, args.segments, args.steps, args.warmup, per_segment=False,
                             count=args.segment_count, tune=not args.no_tune)
        print(json.dumps({"segments": args.segments, **res}), flush=True)
        return

    import torch

    import turbosort_b200 as ts

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist_mod = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    ctx = ts.Context(local)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)

    kind, dist, lg = WORKLOADS[args.workload]
    if args.log2n:
        lg = args.log2n
    # the tile autotuner for the workload's key width (and 8-byte keys for the
    # breakdown), before anything is timed
    if args.no_tune:
        tuning = {str(WIDTH[kind]): {"variants": ctx.lsd_variants(WIDTH[kind]), "tuned": False}}
    else:
        tuning = {str(WIDTH[kind]): ctx.lsd_autotune(WIDTH[kind])}
        if not args.no_breakdown and WIDTH[kind] != 8:
            tuning["8"] = ctx.lsd_autotune(8)
    clocks = Clocks(local)
    clocks.start()
    r = bench_device(ts, torch, ctx, kind, dist, lg, args.steps, args.warmup, 0x9E3779B97F4A7C15 + rank, dist_mod,
                     rank, world)
    clk = clocks.stop()
    ms, r["ok"] = reduce_over_ranks(torch, dist_mod, r["ms_total"], r["ok"], f"cuda:{local}")
    n, w, live = r["n"], r["w"], r["live"]
    ms_step = ms / args.steps
    value = whole_job_gkeys(world, n, ms_step)

    peak, peak_kind = measured_peak_gbs()
    sweep_ms, sweep_count = r["timings"].get("onesweep", (0.0, 0))
    live_launches = max(1, live * args.steps)
    per_launch_ms = sweep_ms / live_launches if sweep_ms else None
    pass_bytes = n * w * 2
    achieved = pass_bytes / (per_launch_ms / 1e3) / 1e9 if per_launch_ms else None
    sort_bytes = sort_bytes_of(r)
    traffic = ncu_traffic(f"onesweep_{kind}_2p{lg}.md")

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "GKeys/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": kind, "data": "synthetic (seeded xorshift64 keys)",
        "config": workload_config(args.workload, lg),
        "bit_exact_checks": ("byte-equal to numpy's sort of the input's radix keys (every workload, full size)"
                             if r["ok"] else "FAILED"),
        "roofline": {
            "bound": "hbm", "kernel": "k_onesweep (one live digit pass)",
            "achieved": round(achieved, 1) if achieved else None, "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4) if achieved else None, "peak_source": peak_kind,
            "traffic": traffic, "algorithmic_bytes_per_launch": pass_bytes,
            "avg_launch_ms": round(per_launch_ms, 4) if per_launch_ms else None,
            "live_passes": live, "divert_shift": r["divert_shift"],
            "sort_bytes": sort_bytes,
            "sort_achieved_gbs": round(sort_bytes / (ms_step / 1e3) / 1e9, 1),
            "sort_frac": round(sort_bytes / (ms_step / 1e3) / 1e9 / peak, 4),
        },
        "kernel_ms_per_step": {k: round(v[0] / args.steps, 4) for k, v in r["timings"].items()},
        "gpu_launches": int(r["launches"]),
        "clocks": clk,
        "tuning": tuning,
    }

    # end to end through the host-slice C ABI call, pinned host memory: the
    # library's default (copies overlapped with chunk sorts and merges), then
    # the same call with the copies serialised, for comparison
    if not args.no_e2e:
        host = gen(kind, dist, n, 0x9E3779B97F4A7C15 + rank)
        pinned = torch.empty(n * w, dtype=torch.uint8, pin_memory=True).numpy().view(NP[kind])
        want = expected_radix(host)

        def host_calls(steps, buf):
            e_ms, ok = [], True
            for i in range(args.warmup + steps):
                np.copyto(buf, host)
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                ts.sort(buf, ctx)
                e1.record()
                torch.cuda.synchronize()
                if i >= args.warmup:
                    e_ms.append(e0.elapsed_time(e1))
            ok = check_exact(buf, want)
            total = sum(e_ms)
            if dist_mod is not None:
                t = torch.tensor([total], dtype=torch.float64, device=f"cuda:{local}")
                dist_mod.all_reduce(t, op=dist_mod.ReduceOp.MAX)
                total = float(t.item())
            return total, ok

        ctx.transfer_pipeline(PIPE_CHUNKS, PIPE_MIN_BYTES)
        emax, ok = host_calls(args.steps, pinned)
        serial_steps = max(1, min(args.steps, 5))
        ctx.transfer_pipeline(1, PIPE_MIN_BYTES)
        smax, sok = host_calls(serial_steps, pinned)
        ctx.transfer_pipeline(PIPE_CHUNKS, PIPE_MIN_BYTES)
        # the same call on pageable host memory (what a Rust &mut [T] usually is)
        del pinned
        pageable = np.empty(n, dtype=NP[kind])
        pmax, pok = host_calls(serial_steps, pageable)
        del pageable
        line["e2e"] = {"value": round(world * n * args.steps / (emax / 1e3) / 1e9, 3), "unit": "GKeys/s",
                       "h2d_bytes_per_step": n * w, "d2h_bytes_per_step": n * w,
                       "ms_per_step": round(emax / args.steps, 3),
                       "call": f"ts_sort_{kind} on pinned host memory",
                       "pipeline": {"chunks": PIPE_CHUNKS, "min_bytes": PIPE_MIN_BYTES,
                                    "serial_ms_per_step": round(smax / serial_steps, 3)},
                       "pageable": {"value": round(world * n * serial_steps / (pmax / 1e3) / 1e9, 3),
                                    "ms_per_step": round(pmax / serial_steps, 3),
                                    "call": f"ts_sort_{kind} on pageable host memory (pinned staging slots)"},
                       "bit_exact_checks": "byte-equal to numpy's sort" if ok and sok and pok else "FAILED"}

    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        rate, sample = cpu_sample_rate(kind, dist, n, 15.0, threads, 0x9E3779B97F4A7C15)
        line["cpu_baseline"] = {"value": round(rate, 4), "unit": "GKeys/s", "cores": threads, "kind": "port",
                                "sample": sample, "cpu": cpu_model(),
                                "what": "turbosort sort_parallel (src/parallel.rs) restated in C, pthreads"}
        rate1, sample1 = cpu_sample_rate(kind, dist, n, 10.0, 1, 0x9E3779B97F4A7C15, serial=True)
        line["cpu_baseline_serial"] = {"value": round(rate1, 4), "unit": "GKeys/s", "cores": 1, "kind": "port",
                                       "sample": sample1, "cpu": cpu_model(),
                                       "what": "turbosort sort (src/lib.rs:99, src/dispatch.rs:31) restated in C, "
                                               "one core"}

    if not args.no_breakdown:
        bd = {}
        for name in [k for k in WORKLOADS if k != args.workload and k != "c1_u32_2p20"]:
            k2, d2, l2 = WORKLOADS[name]
            rr = bench_device(ts, torch, ctx, k2, d2, l2, max(3, args.steps // 2), 3, 0x1234 + rank, None, rank,
                              world)
            st = rr["ms_total"] / max(3, args.steps // 2)
            sb = sort_bytes_of(rr)
            ow = rr["timings"].get("onesweep", (0.0, 0))[0] / max(1, rr["live"] * max(3, args.steps // 2))
            bd[name] = {"gkeys_s": round(rr["n"] / (st / 1e3) / 1e9, 2), "ms": round(st, 4), "live_passes": rr["live"],
                        "divert_shift": rr["divert_shift"],
                        "sort_frac": round(sb / (st / 1e3) / 1e9 / peak, 3),
                        "pass_frac": round(rr["n"] * rr["w"] * 2 / (ow / 1e3) / 1e9 / peak, 3) if ow else None,
                        "ok": rr["ok"]}
        bd["c1_u32_2p20"] = bench_small(ts, torch, ctx, "u32", 0, 20, max(10, args.steps), 5, 0x1234 + rank)
        bd["c1_u32_2p20"]["tier"] = ctx.last_sort_info()["tier"]
        # the same sort through the multi-launch LSD, for comparison
        ctx.set_single_launch(False)
        bd["c1_u32_2p20_multi_launch"] = bench_small(ts, torch, ctx, "u32", 0, 20, max(10, args.steps), 5,
                                                     0x1234 + rank)
        ctx.set_single_launch(True)
        bd["tiny_slices_u32"] = bench_tiny(ts, torch, ctx, max(10, args.steps))
        bd["c3_by_key_zipf_u64_2p27"] = bench_by_key(ts, torch, ctx, 27, max(3, args.steps // 2), 3, peak)
        for kind in ("u32", "f32"):
            bd[f"c4_segments_{kind}"] = bench_segments(ts, torch, ctx, kind, max(3, args.steps // 2), 2)
        for kind in ("lognormal_f64", "gauss_mix_u64", "unit_f32_dups"):
            bd[f"c5_learned_{kind}_2p28"] = bench_learned(ts, torch, ctx, kind, max(3, args.steps // 2), 3, peak)
        line["breakdown"] = bd

    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist_mod is not None:
        dist_mod.barrier()
        dist_mod.destroy_process_group()


if __name__ == "__main__":
    main()
