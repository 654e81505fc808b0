#!/usr/bin/env python
"""Benchmark: GHive's offloaded relational operators on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload (one GPU's worth, weak-scaled over N ranks): the inner hash
equi-join of a 1.5M-row build side (unique int64 keys, int64 + double
payloads) with a 60M-row probe side (int64 foreign key, 5% misses, int32
payload), emitting every (probe row id, build int64 payload, build double
payload) match.  One step = build the table + probe all 60M rows.

Before the headline line (the last line, the only one with "metric"), one
JSON line per further operator workload (single GPU, N = 1 only), each with
its device-timed rows/s, its HBM roofline, a CPU baseline (the C++
restatement of Hive's vectorized operator at T = 1 and T = all host threads)
and an end-to-end figure through the host-buffer entry point:
  - "filter_groupby": filter d < 1263 + GROUP BY k over the 6M-row fact table,
    with the error of each DOUBLE SUM/AVG against an FP64 compensated sum;
  - "join_hashed": the headline join with the keys spread over the int64
    range (the hashed table instead of the direct one);
  - "sort": ORDER BY (d, k) of 60M rows, uniform and Zipf(0.99) k;
  - "batched_groupby": 512 filter + group-by instances in one launch against
    one call per instance;
  - "served_mix": the served mixed operator stream against serial per-call
    execution with the same resident tables and output sets.

Timing: CUDA events on the launching stream, W untimed warm-up steps, then K
timed steps between a barrier + device synchronise on both sides; the
reported time is the max over ranks.  The join's probe key column (480 MB)
and the sort's columns are larger than the 126 MB L2; the group-by step flushes
L2 (a 256 MB write) before each timed launch.  Inputs are seeded PCG64
synthetic data of the workload shapes.

`--impl reference` times the CPU restatement of Hive's vectorized map-join
(the oracle port: HashCodeUtil hash, triangular probing, load factor 0.75)
on all host threads over the same workload: one build + all 60M probe rows
per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_BUILD = 1_500_000
N_PROBE = 60_000_000
N_FACT = 6_000_000
N_SORT = 60_000_000
METRIC = "GPU rows/s (inner hash join: probe rows per second, build + probe per step)"
JOIN_OUTPUT_ROWS = 56_999_683   # matches of the rank-0 probe (seeded), for the shared config


def join_config(world):
    """The workload both arms time (identical dicts, so the arms compare)."""
    return {"workload": "inner hash join, build 1.5M unique int64 keys + int64/double payloads, "
                        "probe 60M int64 keys (5% miss), output (probe row, int64 payload, double "
                        "payload) per match",
            "build_rows": N_BUILD, "probe_rows": N_PROBE, "output_rows": JOIN_OUTPUT_ROWS,
            "parallelism": "dp%d (replicated build, sharded probe, no collective)" % world,
            "l2": "inputs larger than L2 (probe key column 480 MB)"}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name):
    """DRAM bytes per launch recorded in a committed ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":")[1])
    return None


def roofline(nbytes, ms, peak, peak_kind, **extra):
    ach = nbytes / (ms / 1e3) / 1e9
    d = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
         "peak_kind": peak_kind, "bytes_per_launch": int(nbytes), "ms_per_launch": ms}
    d.update(extra)
    return d


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device, self.rows, self.proc = device, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def dist_init(gpus, impl):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and impl == "ours":   # the CPU arm needs no collective
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, v, device):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def timed_cpu(fn):
    t0 = time.perf_counter()
    r = fn()
    return time.perf_counter() - t0, r


def host_threads():
    return os.cpu_count() or 1


# ----------------------------------------------------------------- CPU arm
def run_reference(args, world, rank):
    """The C++ restatement of Hive's map-join (build + probe of all 60M rows
    per step) on every host thread; rank 0 alone runs it."""
    if rank != 0:
        return 0
    from ghive_b200 import workloads
    from oracle import oracle
    threads = host_threads()
    (bkey, bpay), (fk, _) = workloads.join_tables(N_BUILD, N_PROBE, seed_idx=1)
    secs, rows = [], None
    for i in range(args.warmup + args.steps):
        dt, (prow, _) = timed_cpu(lambda: oracle.hash_join_mt(threads, bkey, fk, bpay, cap=N_PROBE))
        rows = len(prow)
        if i >= args.warmup:
            secs.append(dt)
    step_s = statistics.median(secs)
    dt1, _ = timed_cpu(lambda: oracle.hash_join_mt(1, bkey, fk, bpay, cap=N_PROBE))
    value = N_PROBE / step_s
    sample = ("each step: build 1.5M rows + probe all 60M probe rows (Hive "
              "VectorMapJoinFastLongHashTable + VectorMapJoinInnerLongOperator restated in C++), "
              "%d matches; T=1: %.3g rows/s (one step, %.1f s)" % (rows, N_PROBE / dt1, dt1))
    if world > 1:
        sample += "; one rank's 60M-row probe shard per step (every shard has this shape)"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "rows/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded PCG64)",
            "config": join_config(world),
            "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port",
                             "sample": sample, "t1_value": N_PROBE / dt1},
            "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------- GPU arm
def filter_host_chunks(n):
    """Chunks of ghb_filter_host's pipelined path over n pinned rows (one
    int64 row count comes back per chunk): about n/12 rows each, whole
    2048-row tiles between 512Ki and 8Mi rows; below two chunks, one call."""
    c = min(8 << 20, max(512 << 10, (n + 11) // 12))
    c = (c + 2047) // 2048 * 2048
    return (n + c - 1) // c if n >= 2 * c else 1


def pinned(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()


def pinned_outs(types, cap, with_nulls=True):
    """Host output columns in pinned memory (the D2H copies run at DMA speed)."""
    import torch

    from ghive_b200 import abi
    from ghive_b200.ops import _Outs
    o = _Outs(types, cap, None, with_nulls=with_nulls)
    keep = []
    for j, t in enumerate(types):
        buf = torch.empty(max(1, cap), dtype={abi.LONG: torch.int64, abi.DOUBLE: torch.float64,
                                              abi.INT: torch.int32}[t]).pin_memory()
        nb = torch.empty(max(1, cap), dtype=torch.uint8).pin_memory() if with_nulls else None
        o.cols[j] = (buf.numpy(), None if nb is None else nb.numpy())
        o.arr[j].data = buf.data_ptr()
        o.arr[j].is_null = None if nb is None else nb.data_ptr()
        keep += [buf, nb]
    o._pinned = keep
    return o


def probe_outs(types, cap, dev):
    """Device outputs of a probe emitting (probe row id, build payloads)."""
    import torch

    from ghive_b200.ops import _Outs
    ob = _Outs(types, cap, dev, with_nulls=False)
    op = _Outs([], cap, dev)
    prow = torch.empty(cap, dtype=torch.int32, device=dev)
    d_rows = torch.zeros(1, dtype=torch.int64, device=dev)
    return (ob, op, prow, None, d_rows)


def run_ours(args, world, rank, local):
    import torch

    from ghive_b200 import abi, workloads
    from ghive_b200.ops import Context

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = Context(local)
    stream = torch.cuda.current_stream()
    peak, peak_kind = load_peaks()

    # ---------------- headline: hash join, data resident in HBM
    (bkey, bpay), (fk, ppay) = workloads.join_tables(N_BUILD, N_PROBE, seed_idx=1 + 17 * rank)
    d_bkey = torch.from_numpy(bkey).to(dev)
    d_bpay = [torch.from_numpy(c).to(dev) for c in bpay]
    d_fk = torch.from_numpy(fk).to(dev)
    cap = N_PROBE
    outs = probe_outs([abi.LONG, abi.DOUBLE], cap, dev)
    d_rows = outs[4]

    def join_step(ev=None):
        t = ctx.join_build(d_bkey, build_payload=d_bpay)
        if ev:
            ev[0].record(stream)
        ctx.join_probe(t, d_fk, abi.INNER_JOIN, capacity=cap, rowids=False, sync=False, outs=outs)
        if ev:
            ev[1].record(stream)
        t.free()

    for _ in range(args.warmup):
        join_step()
    ctx.sync()
    rows_out = int(d_rows.item())
    probe_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                for _ in range(args.steps)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    l0 = ctx.launches
    with ClockSampler(local) as clk:
        start.record(stream)
        for i in range(args.steps):
            join_step(probe_ev[i])
        end.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    launches = ctx.launches - l0
    ctx.sync()
    step_ms = start.elapsed_time(end) / args.steps
    step_ms = max_over_ranks(world, step_ms, dev)
    probe_ms = statistics.mean(a.elapsed_time(b) for a, b in probe_ev)
    value = world * N_PROBE / (step_ms / 1e3)
    probe_bytes = N_PROBE * 8 + rows_out * 20 + N_BUILD * 16

    # ---------------- e2e: host buffers through the C ABI entry point
    h_bkey, h_bpay, h_fk = pinned(bkey), [pinned(c) for c in bpay], pinned(fk)
    hob = pinned_outs([abi.LONG, abi.DOUBLE], cap, with_nulls=False)
    hop = pinned_outs([], cap)
    hprow = torch.empty(cap, dtype=torch.int32).pin_memory().numpy()
    e2e_steps = max(1, min(args.steps, 5))
    for _ in range(2):
        ctx.hash_join_host(h_bkey, h_fk, abi.INNER_JOIN, build_payload=h_bpay, capacity=cap,
                           outs=(hob, hop, hprow, None))
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        r = ctx.hash_join_host(h_bkey, h_fk, abi.INNER_JOIN, build_payload=h_bpay, capacity=cap,
                               outs=(hob, hop, hprow, None))
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) / e2e_steps * 1e3
    barrier(world)
    e2e_ms = max_over_ranks(world, e2e_ms, dev)
    assert r["rows"] == rows_out
    e2e = {"value": world * N_PROBE / (e2e_ms / 1e3), "unit": "rows/s",
           "h2d_bytes_per_step": int(bkey.nbytes + sum(c.nbytes for c in bpay) + fk.nbytes),
           "d2h_bytes_per_step": int(rows_out * 20 + 8), "ms_per_step": e2e_ms,
           "api": "ghb_hash_join_host (pinned host columns; host clock, returns with the "
                  "results in host memory)"}
    del d_fk, outs
    torch.cuda.empty_cache()

    lines = []
    if world == 1 and not args.headline_only:
        lines.append(bench_filter(ctx, args, dev, stream, peak, peak_kind))
        lines.append(bench_groupby(ctx, args, dev, stream, peak, peak_kind))
        lines.append(bench_join_hashed(ctx, args, dev, stream, peak, peak_kind))
        lines.append(bench_sort(ctx, args, dev, stream, peak, peak_kind))
        if not args.skip_batched:
            lines.append(bench_batched(ctx, args, dev, stream, peak, peak_kind))
        if not args.skip_served:
            lines.append(bench_served(ctx, args, dev))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle
        threads = host_threads()
        dt, _ = timed_cpu(lambda: oracle.hash_join_mt(threads, bkey, fk, bpay, cap=N_PROBE))
        # T=1 on a bounded sample: the build and the first 6M probe rows
        s1 = 6_000_000
        dt1, _ = timed_cpu(lambda: oracle.hash_join_mt(1, bkey, fk[:s1], bpay, cap=s1))
        cpu = {"value": N_PROBE / dt, "unit": "rows/s", "cores": threads, "kind": "port",
               "t1_value": s1 / dt1,
               "sample": "T=all: one full step, build 1.5M rows + probe all 60M probe rows (Hive "
                         "VectorMapJoinFastLongHashTable restated, C++), %.2f s; T=1: the build + "
                         "the first 6M probe rows, %.2f s" % (dt, dt1)}

    if rank == 0:
        for ln in lines:
            print(json.dumps(ln), flush=True)
        cfg = join_config(world)
        cfg["output_rows"] = rows_out if world == 1 else cfg["output_rows"]
        line = {"metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
                "data": "synthetic (seeded PCG64)", "config": cfg,
                "roofline": roofline(probe_bytes, probe_ms, peak, peak_kind,
                                     kernel="join probe: count + scan + write passes (one "
                                            "ghb_join_probe call)",
                                     traffic=profile_traffic("join_probe_60M.md")),
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clk.summary(),
                "ops": [ln["op"] for ln in lines]}
        print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def flush_l2(buf):
    buf.add_(1)


def _double_errors(gpu_keys, gpu_aggs, ok, comp, out_types):
    """Relative error of each DOUBLE SUM/AVG result against the oracle's FP64
    Neumaier compensated sum (groups matched by key)."""
    gk = gpu_keys[0][0].cpu().numpy()
    okk = ok[0][0]
    go, oo = np.argsort(gk, kind="stable"), np.argsort(okk, kind="stable")
    errs = []
    from ghive_b200 import abi
    for j, t in enumerate(out_types):
        if t != abi.DOUBLE or not np.any(comp[j] != 0):
            continue
        g = gpu_aggs[j][0].cpu().numpy()[go]
        c = comp[j][oo]
        errs.append(np.abs(g - c) / np.maximum(np.abs(c), 1e-300))
    e = np.concatenate(errs) if errs else np.zeros(0)
    return {"results": int(e.size), "max_rel": float(e.max()) if e.size else None,
            "median_rel": float(np.median(e)) if e.size else None,
            "reference": "FP64 Neumaier compensated sum per group (CPU oracle)"}


def bench_filter(ctx, args, dev, stream, peak, peak_kind):
    """The filter alone on the fact table: d < 1263 over 6M rows, the four
    columns of each passing row written out in order."""
    import torch

    from ghive_b200 import abi, workloads
    from ghive_b200.ops import _Outs
    cols = workloads.fact_table(N_FACT, seed_idx=0)
    dcols = [torch.from_numpy(c).to(dev) for c in cols]
    pred = workloads.fact_predicate()
    types = [abi.INT, abi.LONG, abi.DOUBLE, abi.INT]
    outs = _Outs(types, N_FACT, dev, with_nulls=False)
    flush = torch.zeros(64 << 20, dtype=torch.float32, device=dev)  # 256 MB
    for _ in range(args.warmup):
        ctx.filter(pred, dcols, outs=outs, sync=False)
    ctx.sync()
    times = []
    for _ in range(max(args.steps, 10)):
        flush_l2(flush)
        torch.cuda._sleep(300_000)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        _, d_rows = ctx.filter(pred, dcols, outs=outs, sync=False)
        b.record(stream)
        times.append((a, b))
    ctx.sync()
    rows = int(d_rows.item())
    ms = statistics.median(x.elapsed_time(y) for x, y in times)
    nbytes = N_FACT * 24 + rows * 24
    # e2e: pinned host columns through ghb_filter_host
    hcols = [pinned(c) for c in cols]
    houts = pinned_outs(types, N_FACT, with_nulls=False)
    ctx.filter_host(pred, hcols, outs=houts)
    t0 = time.perf_counter()
    for _ in range(5):
        ctx.filter_host(pred, hcols, outs=houts)
    e2e_ms = (time.perf_counter() - t0) / 5 * 1e3
    out = {"op": "filter",
           "workload": "filter d<1263 over the 6M-row fact table (k i32, qty i64, price f64, d i32), "
                       "the passing rows' four columns written in order",
           "value": N_FACT / (ms / 1e3), "unit": "rows/s", "ms": ms, "rows_out": rows,
           "roofline": roofline(nbytes, ms, peak, peak_kind,
                                kernel="filter_kernel (per range of tiles: predicate ballots, one look-back, "
                                       "the projected columns' selected rows)",
                                l2="flushed before each launch",
                                traffic=profile_traffic("filter_fact6M.md")),
           "e2e": {"value": N_FACT / (e2e_ms / 1e3), "unit": "rows/s", "ms_per_step": e2e_ms,
                   "h2d_bytes_per_step": int(sum(c.nbytes for c in cols)),
                   "d2h_bytes_per_step": int(rows * 24 + 8 * filter_host_chunks(N_FACT)),
                   "api": "ghb_filter_host (pinned host columns and outputs)"}}
    if not args.no_cpu:
        from oracle import oracle
        import numpy as np

        from concurrent.futures import ThreadPoolExecutor

        def cpu_range(lo, hi):
            part = [c[lo:hi] for c in cols]
            sel = oracle.filter_rows(pred, part)
            return [np.take(c, sel) for c in part]
        t1, _ = timed_cpu(lambda: cpu_range(0, N_FACT))
        threads = host_threads()
        bounds = [(N_FACT * i // threads, N_FACT * (i + 1) // threads) for i in range(threads)]

        def cpu_all():
            with ThreadPoolExecutor(threads) as ex:
                return list(ex.map(lambda b: cpu_range(*b), bounds))
        tn, _ = timed_cpu(cpu_all)
        out["cpu_baseline"] = {"value": N_FACT / tn, "unit": "rows/s", "cores": threads, "kind": "port",
                               "t1_value": N_FACT / t1,
                               "sample": "the whole 6M-row workload: Hive's filter restated in C++ "
                                         "(selected rows), then the projected columns gathered; "
                                         "T=all: row ranges, one per thread"}
    del dcols, flush, outs
    torch.cuda.empty_cache()
    return out


def bench_groupby(ctx, args, dev, stream, peak, peak_kind):
    import torch

    from ghive_b200 import abi, workloads
    cols = workloads.fact_table(N_FACT, seed_idx=0)
    dcols = [torch.from_numpy(c).to(dev) for c in cols]
    pred, aggs = workloads.fact_predicate(), workloads.AGGS_FACT
    out_types = [abi.LONG, abi.LONG, abi.DOUBLE, abi.DOUBLE, abi.INT, abi.INT]
    flush = torch.zeros(64 << 20, dtype=torch.float32, device=dev)  # 256 MB
    res = None
    for _ in range(args.warmup):
        res = ctx.filter_groupby(pred, dcols, [0], aggs, capacity=1000, max_groups=1000, sync=False)
    ctx.sync()
    times = []
    for _ in range(max(args.steps, 10)):
        flush_l2(flush)
        # the GPU stays busy while the host prepares the call, so the events
        # bracket the operator's kernels and not the host's launch latency
        torch.cuda._sleep(300_000)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        res = ctx.filter_groupby(pred, dcols, [0], aggs, capacity=1000, max_groups=1000, sync=False)
        b.record(stream)
        times.append((a, b))
    ctx.sync()
    groups = int(res[1].item())
    ms = statistics.median(x.elapsed_time(y) for x, y in times)
    # the whole call from the host: argument checks, signature lookup, launches
    ctx.sync()
    t0 = time.perf_counter()
    reps = 20
    for _ in range(reps):
        res = ctx.filter_groupby(pred, dcols, [0], aggs, capacity=1000, max_groups=1000, sync=False)
    ctx.sync()
    call_ms = (time.perf_counter() - t0) / reps * 1e3
    gk, ga, _ = ctx.filter_groupby(pred, dcols, [0], aggs, capacity=1000, max_groups=1000)

    # e2e: pinned host columns through ghb_filter_groupby_host
    hcols = [pinned(c) for c in cols]
    houts = pinned_outs([abi.INT] + out_types, 1000)   # key k (int32), then the aggregates
    ctx.filter_groupby_host(pred, hcols, [0], aggs, 1000, max_groups=1000, outs=houts)
    t0 = time.perf_counter()
    for _ in range(5):
        ctx.filter_groupby_host(pred, hcols, [0], aggs, 1000, max_groups=1000, outs=houts)
    e2e_ms = (time.perf_counter() - t0) / 5 * 1e3

    out = {"op": "filter_groupby",
           "workload": "filter d<1263 + GROUP BY k (1000 groups): COUNT(*), SUM(qty), SUM(price), "
                       "AVG(price), MIN(d), MAX(d) over 6M rows",
           "value": N_FACT / (ms / 1e3), "unit": "rows/s", "ms": ms, "groups": groups,
           "host_call_ms": call_ms,
           "roofline": roofline(N_FACT * 24 + groups * 48, ms, peak, peak_kind,
                                kernel="fold + finalize (one ghb_filter_groupby call)",
                                l2="flushed before each launch",
                                traffic=profile_traffic("groupby_fold_fact6M.md")),
           "e2e": {"value": N_FACT / (e2e_ms / 1e3), "unit": "rows/s", "ms_per_step": e2e_ms,
                   "h2d_bytes_per_step": int(sum(c.nbytes for c in cols)),
                   "d2h_bytes_per_step": int(groups * 44 + 8),
                   "api": "ghb_filter_groupby_host (pinned host columns)"}}
    if not args.no_cpu:
        from oracle import oracle
        threads = host_threads()
        t1, _ = timed_cpu(lambda: oracle.filter_groupby(pred, cols, [0], aggs, cap=1000))
        tn, _ = timed_cpu(lambda: oracle.filter_groupby(pred, cols, [0], aggs, cap=1000,
                                                        threads=threads))
        out["cpu_baseline"] = {"value": N_FACT / tn, "unit": "rows/s", "cores": threads,
                               "kind": "port", "t1_value": N_FACT / t1,
                               "sample": "the whole 6M-row workload (Hive VectorFilterOperator + "
                                         "VectorGroupByOperator hash mode restated in C++, 1024-row "
                                         "batches); T=all: row ranges with private hash maps, merged"}
        # the checker: the oracle's compensated sums beside the GPU's results
        ok, oa, comp = oracle.filter_groupby(pred, cols, [0], aggs, cap=1000, with_comp=True)
        out["double_error_vs_compensated_sum"] = _double_errors(gk, ga, ok, comp, out_types)
    # Hive's layout: every integer column 8 bytes wide (k and d as int64)
    wcols = [dcols[0].to(torch.int64), dcols[1], dcols[2], dcols[3].to(torch.int64)]
    for _ in range(args.warmup):
        res = ctx.filter_groupby(pred, wcols, [0], aggs, capacity=1000, max_groups=1000, sync=False)
    ctx.sync()
    times = []
    for _ in range(max(args.steps, 10)):
        flush_l2(flush)
        torch.cuda._sleep(300_000)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        res = ctx.filter_groupby(pred, wcols, [0], aggs, capacity=1000, max_groups=1000, sync=False)
        b.record(stream)
        times.append((a, b))
    ctx.sync()
    wms = statistics.median(x.elapsed_time(y) for x, y in times)
    wgroups = int(res[1].item())
    out["hive_layout"] = {"workload": "the same query with k and d as int64 (32 B/row read)",
                          "value": N_FACT / (wms / 1e3), "unit": "rows/s", "ms": wms, "groups": wgroups,
                          "roofline": roofline(N_FACT * 32 + wgroups * 48, wms, peak, peak_kind,
                                               kernel="fold + finalize (one ghb_filter_groupby call)",
                                               l2="flushed before each launch")}
    del dcols, wcols, flush
    torch.cuda.empty_cache()
    return out


def bench_join_hashed(ctx, args, dev, stream, peak, peak_kind):
    """The headline join with keys spread over the int64 range: the hashed
    table layout (bucketized open addressing) instead of the direct one."""
    import torch

    from ghive_b200 import abi, workloads
    (bkey, bpay), (fk, _) = workloads.join_tables(N_BUILD, N_PROBE, seed_idx=1, sparse=True)
    d_bkey = torch.from_numpy(bkey).to(dev)
    d_bpay = [torch.from_numpy(c).to(dev) for c in bpay]
    d_fk = torch.from_numpy(fk).to(dev)
    outs = probe_outs([abi.LONG, abi.DOUBLE], N_PROBE, dev)
    t = ctx.join_build(d_bkey, build_payload=d_bpay)
    for _ in range(args.warmup):
        ctx.join_probe(t, d_fk, abi.INNER_JOIN, capacity=N_PROBE, rowids=False, sync=False,
                       outs=outs)
    ctx.sync()
    ev = []
    for _ in range(max(3, min(args.steps, 10))):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx.join_probe(t, d_fk, abi.INNER_JOIN, capacity=N_PROBE, rowids=False, sync=False,
                       outs=outs)
        b.record(stream)
        ev.append((a, b))
    ctx.sync()
    rows_out = int(outs[4].item())
    _, _, slots = t.info()
    t.free()
    ms = statistics.mean(a.elapsed_time(b) for a, b in ev)
    nbytes = N_PROBE * 8 + rows_out * 20 + N_BUILD * 16
    del d_fk, outs
    torch.cuda.empty_cache()
    return {"op": "join_hashed",
            "workload": "the headline join (1.5M x 60M) with every key passed through a 64-bit "
                        "bijection (keys spread over the int64 range): hashed table, %d slots"
                        % slots,
            "value": N_PROBE / (ms / 1e3), "unit": "rows/s", "ms": ms, "output_rows": rows_out,
            "roofline": roofline(nbytes, ms, peak, peak_kind,
                                 kernel="join probe on the hashed table (count + scan + write)",
                                 traffic=profile_traffic("join_probe_hashed_60M.md"))}


def bench_sort(ctx, args, dev, stream, peak, peak_kind):
    import torch

    from ghive_b200 import abi, workloads
    out = {"op": "sort",
           "workload": "ORDER BY (d int32, k int64) ASC, stable, int32 row-id payload, 60M rows"}
    for zipf in (False, True):
        d, k, rowid = workloads.sort_table(N_SORT, zipf=zipf, seed_idx=2)
        dd, dk, dr = (torch.from_numpy(x).to(dev) for x in (d, k, rowid))
        # the outputs (d, k, row id; the inputs hold no NULLs, so no NULL maps)
        # made once, as the join's are
        from ghive_b200.ops import _Outs
        souts = (_Outs([abi.INT, abi.LONG], N_SORT, dev, with_nulls=False),
                 _Outs([abi.INT], N_SORT, dev, with_nulls=False))
        for _ in range(max(1, args.warmup)):
            ctx.sort([dd, dk], payload=[dr], sync=False, outs=souts)
        ctx.sync()
        l0 = ctx.launches
        ctx.sort([dd, dk], payload=[dr], sync=False, outs=souts)
        ctx.sync()
        # the sort launches a min/max and a histogram kernel, then one kernel
        # per executed radix pass
        passes = ctx.launches - l0 - 2
        times = []
        for _ in range(max(3, min(args.steps, 10))):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            ctx.sort([dd, dk], payload=[dr], sync=False, outs=souts)
            b.record(stream)
            times.append((a, b))
        ctx.sync()
        ms = statistics.median(x.elapsed_time(y) for x, y in times)
        per_pass_bytes = N_SORT * 12 + passes * N_SORT * 24 + N_SORT * 16
        # e2e: pinned host columns through ghb_sort_host
        hd, hk, hr = pinned(d), pinned(k), pinned(rowid)
        hok = pinned_outs([abi.INT, abi.LONG], N_SORT, with_nulls=False)
        hop = pinned_outs([abi.INT], N_SORT, with_nulls=False)
        ctx.sort_host([hd, hk], payload=[hr], outs=(hok, hop, None))
        t0 = time.perf_counter()
        for _ in range(3):
            ctx.sort_host([hd, hk], payload=[hr], outs=(hok, hop, None))
        e2e_ms = (time.perf_counter() - t0) / 3 * 1e3
        entry = {"value": N_SORT / (ms / 1e3), "unit": "rows/s", "ms": ms, "passes": passes,
                 "roofline": roofline(N_SORT * 32, ms, peak, peak_kind,
                                      kernel="whole sort against the 32 B/row lower bound "
                                             "(read d 4 + k 8 + rowid 4, write 16)"),
                 "roofline_per_pass_formula": roofline(
                     per_pass_bytes, ms, peak, peak_kind,
                     kernel="whole sort against N*12 + P*N*24 + N*16 bytes, P = %d executed "
                            "radix passes" % passes,
                     traffic=profile_traffic("sort_passes_20M.md")),
                 "e2e": {"value": N_SORT / (e2e_ms / 1e3), "unit": "rows/s", "ms_per_step": e2e_ms,
                         "h2d_bytes_per_step": N_SORT * 16, "d2h_bytes_per_step": N_SORT * 16,
                         "api": "ghb_sort_host (pinned host columns)"}}
        if not args.no_cpu:
            from oracle import oracle
            threads = host_threads()
            tn, _ = timed_cpu(lambda: oracle.sort_perm([d, k], threads=threads))
            s1 = 6_000_000
            t1, _ = timed_cpu(lambda: oracle.sort_perm([d[:s1], k[:s1]]))
            entry["cpu_baseline"] = {"value": N_SORT / tn, "unit": "rows/s", "cores": threads,
                                     "kind": "port", "t1_value": s1 / t1,
                                     "sample": "T=all: the whole 60M rows (std::stable_sort per "
                                               "thread chunk + stable merges, BinarySortable "
                                               "order); T=1: the first 6M rows"}
        out["zipf" if zipf else "uniform"] = entry
        del dd, dk, dr
        torch.cuda.empty_cache()
    out["value"] = min(out["uniform"]["value"], out["zipf"]["value"])
    out["unit"] = "rows/s"
    return out


def bench_batched(ctx, args, dev, stream, peak, peak_kind, count=512):
    """512 filter + group-by instances of uneven size: one captured batch vs
    one ghb_filter_groupby call per instance on the same GPU."""
    import ctypes as C

    import torch

    from ghive_b200 import abi, workloads
    from ghive_b200._lib import lib
    from ghive_b200.ops import _Cols, _pred

    specs = workloads.batched_specs(count, seed_idx=3)
    inst = workloads.batched_instances_device(specs, dev)
    rows = sum(s["rows"] for s in specs)
    aggs = workloads.AGGS_FACT
    entries = [(workloads.batched_predicate(s["cut"]), it["cols"],
                max(1, min(s["groups"], s["rows"])) + 8, s["groups"]) for s, it in zip(specs, inst)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b = ctx.batch_groupby(entries, [0], aggs, autotune=True)
    create_s = time.perf_counter() - t0

    def timed(fn, reps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(reps):
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            e.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(e))
        return statistics.median(ms)

    l0 = ctx.launches
    b.launch()
    ctx.sync()
    batch_launches = ctx.launches - l0
    batched_ms = timed(b.launch, max(3, min(args.steps, 10)))
    ctx.sync()
    counts = b.groups.cpu().numpy().copy()

    # one call per instance through the C ABI, arguments prepared beforehand
    # so the loop measures the calls, not Python
    calls = []
    for i, (pred, cols, cap, mg) in enumerate(entries):
        cs = _Cols(cols)
        pp, pk = _pred(pred)
        cfg = abi.GroupByCfg()
        cfg.max_groups = mg
        ka = (C.c_int32 * 1)(0)
        ag = (abi.AggDesc * len(aggs))()
        for j, (t, c) in enumerate(aggs):
            ag[j].type, ag[j].col = t, c
        d_groups = torch.zeros(1, dtype=torch.int64, device=dev)
        calls.append(((ctx.h, pp, cs.ptr, cs.n, ka, 1, ag, len(aggs), b.outs[i].ptr, cap,
                       d_groups.data_ptr(), C.byref(cfg), stream.cuda_stream),
                      (cs, pk, cfg, ka, ag, d_groups)))
    fgb = lib().ghb_filter_groupby

    def per_call(sync):
        for a, _ in calls:
            st = fgb(*a)
            if st:
                raise RuntimeError("ghb_filter_groupby failed: %d" % st)
            if sync:
                ctx.sync()   # a task reads its result before the next call

    l0 = ctx.launches
    per_call(False)
    ctx.sync()
    call_launches = ctx.launches - l0
    async_ms = timed(lambda: per_call(False), 3)
    sync_ms = timed(lambda: per_call(True), 3)
    ctx.sync()
    single_counts = np.array([int(k[-1].item()) for _, k in calls])
    parity = bool(np.array_equal(counts, single_counts))
    b.launch()
    ctx.sync()

    groups = int(counts.sum())
    nbytes = rows * 28 + groups * 52
    out = {"op": "batched_groupby",
           "workload": "%d filter + GROUP BY instances, rows log-U[1e3,1e7] (%d in all), groups "
                       "log-U[10,1e6], Zipf keys, selectivity U[0.01,0.9]; fact-table aggregates"
                       % (count, rows),
           "value": rows / (batched_ms / 1e3), "unit": "rows/s",
           "instances": count, "rows": rows, "groups": groups,
           "batched": {"ms": batched_ms, "rows_per_s": rows / (batched_ms / 1e3),
                       "launches_per_run": batch_launches,
                       "roofline": roofline(nbytes, batched_ms, peak, peak_kind,
                                            l2="inputs (%.1f GB) larger than L2" % (rows * 28 / 1e9))},
           "per_call_sync": {"ms": sync_ms, "rows_per_s": rows / (sync_ms / 1e3)},
           "per_call_async": {"ms": async_ms, "rows_per_s": rows / (async_ms / 1e3),
                              "launches_per_run": call_launches},
           "speedup_vs_per_call_sync": sync_ms / batched_ms,
           "speedup_vs_per_call_async": async_ms / batched_ms,
           "group_counts_equal_per_call": parity,
           "create_s": create_s, "plan": b.describe()}
    if not args.no_cpu:
        # CPU baseline and the double-error check on a bounded sample: the
        # first 64 instances, each run by the sequential oracle (Hive order),
        # the instances spread over every host thread
        from concurrent.futures import ThreadPoolExecutor

        from oracle import oracle
        threads = host_threads()
        sample = list(range(64))
        hcols = [[c.cpu().numpy() for c in inst[i]["cols"]] for i in sample]
        srows = sum(specs[i]["rows"] for i in sample)

        def one(j):
            i = sample[j]
            return oracle.filter_groupby(workloads.batched_predicate(specs[i]["cut"]), hcols[j], [0],
                                         aggs, cap=entries[i][2], with_comp=True)

        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            res = list(ex.map(one, range(len(sample))))
        dt = time.perf_counter() - t0
        # T=1: the first eight of those instances one after the other
        t0 = time.perf_counter()
        for j in range(8):
            one(j)
        dt1 = time.perf_counter() - t0
        rows1 = sum(specs[sample[j]]["rows"] for j in range(8))
        errs = []
        types = [abi.LONG, abi.LONG, abi.DOUBLE, abi.DOUBLE, abi.INT, abi.INT]
        for j, i in enumerate(sample):
            gk, ga, _ = b.results(i, counts)
            e = _double_errors(gk, ga, res[j][0], res[j][2], types)
            if e["results"]:
                errs.append((e["max_rel"], e["results"]))
        out["cpu_baseline"] = {"value": srows / dt, "unit": "rows/s", "cores": threads,
                               "kind": "port", "t1_value": rows1 / dt1,
                               "sample": "instances 0-63 (%d rows), one sequential Hive group-by "
                                         "restatement per instance over a %d-thread pool; T=1: "
                                         "instances 0-7 (%d rows) one after the other"
                                         % (srows, threads, rows1)}
        out["double_error_vs_compensated_sum"] = {
            "results": int(sum(n for _, n in errs)),
            "max_rel": max(m for m, _ in errs) if errs else None,
            "sample": "instances 0-63"}
    b.free()
    del inst, entries, calls
    torch.cuda.empty_cache()
    return out


def bench_served(ctx, args, dev, n_req=300, max_rows=100_000_000, loads=(0.5, 0.8, 0.95)):
    """Served mixed operator stream against serial per-call execution with the
    same resident tables and the same output sets."""
    import itertools
    from concurrent.futures import ThreadPoolExecutor

    import torch

    from ghive_b200 import abi, workloads
    from ghive_b200.serve import Server

    g = torch.Generator(device=dev)
    g.manual_seed(workloads.SEED + 4)

    def ri(lo, hi, n, dt):
        return torch.randint(lo, hi, (n,), generator=g, device=dev, dtype=dt)

    # resident column pools (requests are slices) and 8 build tables
    fact = [ri(0, 1000, max_rows, torch.int32), ri(1, 51, max_rows, torch.int64),
            ri(90000, 10500001, max_rows, torch.int64).to(torch.float64) / 100.0,
            ri(0, 2526, max_rows, torch.int32)]
    sortc = [ri(0, 2526, max_rows, torch.int32), ri(0, 1 << 40, max_rows, torch.int64),
             torch.arange(max_rows, dtype=torch.int32, device=dev)]
    sizes = [int(x) for x in np.exp(workloads.rng(4, 1).uniform(np.log(1e5), np.log(1e7), 8))]
    builds, probes = [], []
    for sz in sizes:
        key = torch.randperm(sz, generator=g, device=dev, dtype=torch.int64) + 1
        builds.append((key, [ri(0, 1 << 62, sz, torch.int64),
                             torch.rand(sz, generator=g, device=dev, dtype=torch.float64)]))
        pk = ri(1, sz + 1, max_rows, torch.int64)
        miss = torch.rand(max_rows, generator=g, device=dev) < 0.05
        probes.append(torch.where(miss, pk + sz, pk))
    specs = workloads.served_specs(n_req, seed_idx=4, max_rows=max_rows)
    rows_total = sum(s["rows"] for s in specs)
    aggs = workloads.AGGS_FACT

    def sl(cols, s):
        return [c[s["offset"]:s["offset"] + s["rows"]] for c in cols]

    # serial per-call execution with what the server has: the 8 build tables
    # resident (built once, outside the timing) and each probe emitting (probe
    # row id, build payloads) without build row ids, as a served probe does
    tables = [ctx.join_build(k, build_payload=p) for k, p in builds]
    pouts = probe_outs([abi.LONG, abi.DOUBLE], max_rows, dev)

    def run_plain(s):
        pred = workloads.fact_predicate(s["cut"])
        if s["op"] == "groupby":
            ctx.filter_groupby(pred, sl(fact, s), [0], aggs, capacity=1000, max_groups=1000)
        elif s["op"] == "filter":
            ctx.filter(pred, sl(fact, s), proj=[0, 1, 2])
        elif s["op"] == "sort":
            ctx.sort(sl(sortc[:2], s), payload=sl(sortc[2:], s))
        else:
            ctx.join_probe(tables[s["table"]], sl([probes[s["table"]]], s)[0], abi.INNER_JOIN,
                           capacity=s["rows"], rowids=False, outs=pouts, sync=False)
            ctx.sync()

    # a full untimed pass first so the allocators hold their sizes
    for s in specs:
        run_plain(s)
    torch.cuda.synchronize()
    service = []
    t0 = time.perf_counter()
    for s in specs:
        a = time.perf_counter()
        run_plain(s)
        service.append(time.perf_counter() - a)
    serial_s = time.perf_counter() - t0
    serial_rate = len(specs) / serial_s
    for t in tables:
        t.free()
    del pouts

    srv = Server(dev.index, slots=8)
    try:
        tids = [srv.add_join_table(k, p) for k, p in builds]

        def submit(i):
            s = specs[i]
            pred = workloads.fact_predicate(s["cut"])
            if s["op"] == "groupby":
                return srv.submit_groupby(pred, sl(fact, s), [0], aggs, 1000)
            if s["op"] == "filter":
                return srv.submit_filter(pred, sl(fact, s), proj=[0, 1, 2])
            if s["op"] == "sort":
                return srv.submit_sort(sl(sortc[:2], s), payload=sl(sortc[2:], s))
            return srv.submit_join(tids[s["table"]], sl([probes[s["table"]]], s)[0])

        def closed(clients):
            it = itertools.count()
            lat = [0.0] * len(specs)

            def client():
                while True:
                    i = next(it)
                    if i >= len(specs):
                        return
                    t = submit(i)
                    try:
                        lat[i] = srv.wait(t).latency_ms
                    finally:
                        srv.release(t)

            a = time.perf_counter()
            ths = [threading.Thread(target=client) for _ in range(clients)]
            for th in ths:
                th.start()
            for th in ths:
                th.join()
            return time.perf_counter() - a, lat

        def pct(v):
            v = np.asarray(v)
            return {"p50_ms": float(np.percentile(v, 50)), "p95_ms": float(np.percentile(v, 95)),
                    "p99_ms": float(np.percentile(v, 99))}

        closed(64)   # warm-up: slot arenas grow to their working sizes
        sat = {}
        for c in (1, 8, 64):
            dt, lat = closed(c)
            sat["clients_%d" % c] = dict(rows_per_s=rows_total / dt, ms=dt * 1e3, **pct(lat))
        best = max(v["rows_per_s"] for v in sat.values())

        load = {}
        arr_rng = workloads.rng(4, 2)
        for frac in loads:
            rate = frac * serial_rate
            arrivals = np.cumsum(arr_rng.exponential(1.0 / rate, len(specs)))
            lat = [0.0] * len(specs)
            qwait = [0.0] * len(specs)
            first, last = [None], [0]

            def waiter(i, t):
                try:
                    r = srv.wait(t)
                    lat[i] = r.latency_ms
                    qwait[i] = (r.admit_ns - r.submit_ns) / 1e6
                    last[0] = max(last[0], r.done_ns)
                    if first[0] is None or r.submit_ns < first[0]:
                        first[0] = r.submit_ns
                finally:
                    srv.release(t)

            with ThreadPoolExecutor(64) as ex:
                a = time.perf_counter()
                futs = []
                for i, at in enumerate(arrivals):
                    d = a + at - time.perf_counter()
                    if d > 0:
                        time.sleep(d)
                    futs.append(ex.submit(waiter, i, submit(i)))
                for f in futs:
                    f.result()
            span = (last[0] - first[0]) / 1e9
            # serial execution under the same arrivals: a FIFO single server with
            # the service times measured above
            fin, slat = 0.0, []
            for at, sv in zip(arrivals, service):
                fin = max(at, fin) + sv
                slat.append((fin - at) * 1e3)
            name = "%d%%" % round(frac * 100)
            load[name] = {
                "offered_requests_per_s": rate,
                "served": dict(rows_per_s=rows_total / span, queue_wait_p50_ms=float(np.median(qwait)),
                               queue_wait_p99_ms=float(np.percentile(qwait, 99)), **pct(lat)),
                "serial": dict(rows_per_s=rows_total / max(fin, 1e-9), **pct(slat))}
    finally:
        srv.close()
    out = {"op": "served_mix",
           "workload": "%d requests: 40%% filter+group-by, 30%% join probe against 8 resident build "
                       "tables (1e5-1e7 keys), 20%% sort, 10%% filter; rows log-U[1e4,1e8] "
                       "(%d in all), device-resident inputs" % (n_req, rows_total),
           "value": best, "unit": "rows/s",
           "requests": n_req, "rows": rows_total, "slots": 8,
           "serial": {"rows_per_s": rows_total / serial_s, "ms": serial_s * 1e3,
                      "note": "one plain operator call at a time, each synchronised; the same "
                              "resident build tables and probe output set as the server"},
           "served_saturation": sat, "speedup_vs_serial": best / (rows_total / serial_s),
           "latency_under_load": load}
    del fact, sortc, builds, probes
    torch.cuda.empty_cache()
    return out


def run_profile_case(case, reps):
    """A small fixed case of one operator's kernels (inputs built on cuda:0,
    the operator run `reps` times so a capture can skip the first, cold
    launch), for ncu captures:

      filter   filter d < 1263 over the 6M-row fact table, four columns out
      groupby  filter d < 1263 + GROUP BY k over the 6M-row fact table
      gbcnt    the same table, COUNT(*) only
      gbrows   GROUP BY k over 1 and then 6M rows of that table: COUNT(*) with
               no predicate, then the filter and the fact aggregates (the
               cost of a call against its rows)
      join     1.5M-key build, 20M-row probe, int64 + double build payloads
      joinhash the same with the keys spread over the int64 range (hashed table)
      sort     ORDER BY (d int32, k int64) with an int32 row id, 20M rows
      batch    64 batched filter + group-by instances (rows log-U[1e3, 2e6])
    """
    import torch

    from ghive_b200 import abi, workloads
    from ghive_b200.ops import Context
    ctx = Context(0)
    dev = torch.device("cuda", 0)
    if case in ("join", "joinhash"):
        (bkey, bpay), (fk, _) = workloads.join_tables(N_BUILD, 20_000_000, seed_idx=1,
                                                      sparse=case == "joinhash")
        db = torch.from_numpy(bkey).to(dev)
        dp = [torch.from_numpy(c).to(dev) for c in bpay]
        df = torch.from_numpy(fk).to(dev)
        outs = probe_outs([abi.LONG, abi.DOUBLE], 20_000_000, dev)
        t = ctx.join_build(db, build_payload=dp)
        for _ in range(reps):
            ctx.join_probe(t, df, abi.INNER_JOIN, capacity=20_000_000, rowids=False, outs=outs)
        print("rows", int(outs[4].item()))
    elif case == "filter":
        cols = [torch.from_numpy(c).to(dev) for c in workloads.fact_table(N_FACT, seed_idx=0)]
        for _ in range(reps):
            _, k = ctx.filter(workloads.fact_predicate(), cols, with_nulls=False)
        print("rows", k)
    elif case in ("groupby", "gbcnt"):
        cols = [torch.from_numpy(c).to(dev) for c in workloads.fact_table(N_FACT, seed_idx=0)]
        aggs = workloads.AGGS_FACT if case == "groupby" else [(abi.CNT, -1)]
        for _ in range(reps):
            _, _, g = ctx.filter_groupby(workloads.fact_predicate(), cols, [0], aggs, capacity=1000,
                                         max_groups=1000)
        print("groups", g)
    elif case == "gbrows":
        big = [torch.from_numpy(c).to(dev) for c in workloads.fact_table(N_FACT, seed_idx=0)]
        for n in (1, N_FACT):
            cols = [c[:n] for c in big]
            for pred, aggs in ((None, [(abi.CNT, -1)]), (workloads.fact_predicate(), workloads.AGGS_FACT)):
                for _ in range(reps):
                    _, _, g = ctx.filter_groupby(pred, cols, [0], aggs, capacity=1000, max_groups=1000)
        print("groups", g)
    elif case == "sort":
        d, k, r = workloads.sort_table(20_000_000, seed_idx=2)
        dd, dk, dr = (torch.from_numpy(x).to(dev) for x in (d, k, r))
        for _ in range(reps):
            ctx.sort([dd, dk], payload=[dr], with_nulls=False)
        print("sorted")
    elif case == "batch":
        specs = workloads.batched_specs(64, seed_idx=3, max_rows=2_000_000)
        inst = workloads.batched_instances_device(specs, dev)
        entries = [(workloads.batched_predicate(s["cut"]), it["cols"],
                    max(1, min(s["groups"], s["rows"])) + 8, s["groups"]) for s, it in zip(specs, inst)]
        b = ctx.batch_groupby(entries, [0], workloads.AGGS_FACT, autotune=False, use_graph=False)
        for _ in range(reps):
            b.launch()
        ctx.sync()
        print("rows", sum(s["rows"] for s in specs))
    else:
        raise SystemExit("unknown profile case %r" % case)
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--profile-case", default=None,
                    help="run one small fixed operator case for an ncu capture and exit")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--headline-only", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--skip-batched", action="store_true")
    ap.add_argument("--skip-served", action="store_true")
    args = ap.parse_args()
    if args.profile_case:
        return run_profile_case(args.profile_case, args.reps)
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_init(args.gpus, args.impl)
    try:
        if args.impl == "reference":
            return run_reference(args, world, rank)
        return run_ours(args, world, rank, local)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
