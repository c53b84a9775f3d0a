"""Benchmark of the full-sort path: ORDER BY of a 50,000,000-row table on one B200 (per GPU).

Workload (one step): a table of 3 columns -- key int64 uniform in [0, 2^40) with a 10% Bernoulli null
bitmap, payload float64 ~ N(0, 1), payload int32 uniform -- sorted by key ascending, nulls last, stable,
then the table taken through the permutation. It runs through the library's C ABI the way the DataFusion
rule calls it: am_plan_run of select_all(sort(scan)). With the table in HBM the payload columns ride
through the sort in row records and the key column comes out of the sort rebuilt from its keys; with
host inputs still uploading, the payload is gathered through the permutation after the sort. Inputs are
seeded synthetic data of the benchmark's shape (numpy default_rng).

  value    rows/s with the table already in HBM: K steps timed with CUDA events on the library's stream
           (no per-launch events), max over ranks; inputs (400 MB key column) are larger than L2, so no
           flush is needed. The per-kernel split comes from a second, profiled loop.
  e2e      the same through the C ABI with host buffers: am_import of the 3 columns from pinned host
           memory (host to device), the plan, am_export of the 3 result columns (device to host); steps
           pipelined two deep in one thread (step i + 1 imported and planned before step i is exported:
           uploads overlap the previous step's downloads), the time one step at a time beside it
           (--e2e-inflight 1: one at a time only).
  roofline the dominant kernel's algorithmic bytes / its CUDA-event time, against the measured HBM
           copy peak.
  cpu_baseline  the CPU oracle (the reference algorithm restated in C) on the host's cores; beside it
           pyarrow's sort_indices + take and DataFusion (when importable).
  full_range, multikey, batched, served  the benchmark's other configurations, each with its own
           CUDA events and clock record (one GPU; --headline-only skips them).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload NAME]
Multi-GPU (torchrun, one rank per GPU) runs independent replicas of the workload: the sort shards by
table / request, with no collective on the data path ("scaling": "weak").
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_ROWS = 50_000_000
SEED = 20260906 + 2
SAT_REPS = 3            # serving: timed repetitions of each saturation run (the best one counts)
METRIC = "rows/s + % HBM peak, 50M int64 argsort+take; batched vs plain; p99 latency"
WORKLOAD = ("ORDER BY int64 key NULLS LAST + take of 3 columns (key int64 uniform [0,2^40) with 10% nulls, "
            "float64 N(0,1), int32 uniform), 50,000,000 rows per GPU")


def make_table(n, seed=SEED):
    rng = np.random.default_rng(seed)
    key = rng.integers(0, 2**40, n, dtype=np.int64)
    valid = rng.random(n) >= 0.10
    p1 = rng.standard_normal(n)
    p2 = rng.integers(-2**31, 2**31 - 1, n, dtype=np.int32, endpoint=True)
    return key, valid, p1, p2


def make_full_range_keys(n, seed=SEED - 1):
    """1,000,000 int64 keys uniform over the whole int64 range, no nulls (the single-key scale case)."""
    rng = np.random.default_rng(seed)
    return rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, n, dtype=np.int64, endpoint=True)


def make_multikey_table(n, seed=SEED + 1):
    """The multi-key case: key1 int32 from 200 distinct values drawn by a bounded Zipf(s=1.1) over their
    ranks (sorted descending); key2 float64 ~ N(0, 1e6) with 0.5% each of -0.0 / +0.0 / +inf / -inf,
    1% NaN and 5% nulls (ascending); a float64 payload ~ N(0, 1)."""
    rng = np.random.default_rng(seed)
    distinct = (rng.choice(2**32, 200, replace=False) - 2**31).astype(np.int32)
    p = np.arange(1, 201, dtype=np.float64) ** -1.1
    key1 = distinct[rng.choice(200, n, p=p / p.sum())]
    key2 = rng.normal(0.0, 1e6, n)
    pos = rng.permutation(n)
    start = 0
    for value, frac in ((-0.0, 0.005), (0.0, 0.005), (np.inf, 0.005), (-np.inf, 0.005), (np.nan, 0.01)):
        cnt = int(n * frac)
        key2[pos[start:start + cnt]] = value
        start += cnt
    valid2 = rng.random(n) >= 0.05
    payload = rng.standard_normal(n)
    return key1, key2, valid2, payload


SEGMENTS = 2048


def make_segments(count=SEGMENTS, seed=SEED + 2):
    """The segmented case: `count` independent arrays with lengths log-uniform in [1e3, 1e6]; even ones
    int64 uniform over the whole range, odd ones float32 ~ N(0, 1) with 2% nulls."""
    import pyarrow as pa
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(10 ** rng.uniform(3, 6)))
        if i % 2 == 0:
            out.append(pa.array(rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, n, dtype=np.int64,
                                             endpoint=True)))
        else:
            out.append(pa.array(rng.standard_normal(n).astype(np.float32), mask=rng.random(n) < 0.02))
    return out


def run_segmented(args, am, torch, stream, local, emit=True):
    """2,048 arrays sorted by one am_argsort_batch call per step, against the same arrays sorted by 2,048
    plain am_argsort_ex2 calls per step (same library, same stream); device time by CUDA events."""
    arrays = make_segments()
    rows = sum(len(a) for a in arrays)
    handles = [am.MetalArray.from_arrow(a) for a in arrays]

    def batched():
        outs = am.argsort_batch(handles)
        del outs

    def plain():
        outs = [h.argsort() for h in handles]
        del outs

    def timed(fn, steps):
        for _ in range(max(args.warmup, 3)):
            fn()
        am.synchronize()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            fn()
        ev1.record(stream)
        ev1.synchronize()
        am.synchronize()
        return ev0.elapsed_time(ev1) / steps

    steps = max(1, min(args.steps, 20))
    with ClockSampler(local) as clocks:
        ms_batched = timed(batched, steps)
        ms_plain = timed(plain, steps)
    am.profile(True)
    am.profile_reset()
    batched()
    am.synchronize()
    prof = am.profile_entries()
    am.profile(False)

    # End to end through the C ABI: host arrays in, host indices out.
    e2e = []
    for i in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hs = [am.MetalArray.from_arrow(a) for a in arrays]
        outs = [o.to_arrow() for o in am.argsort_batch(hs)]
        e2e.append(time.perf_counter() - t0)
        del hs, outs
    e2e_ms = 1e3 * statistics.median(e2e[1:])
    h2d = sum(sum(b.size for b in a.buffers() if b is not None) for a in arrays)
    line = {
        "metric": METRIC, "value": rows / (ms_batched / 1e3), "unit": "rows/s", "n_gpus": 1, "steps": steps,
        "warmup": args.warmup, "ms_per_step": ms_batched, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64/float32", "data": "synthetic",
        "config": {"workload": f"segmented argsort of {len(arrays):,} arrays, lengths log-uniform in [1e3, 1e6] "
                               f"({rows:,} rows), int64 full range and float32 N(0,1) with 2% nulls alternating",
                   "rows": rows, "arrays": len(arrays), "l2": "inputs larger than L2, no flush"},
        "plain": {"value": rows / (ms_plain / 1e3), "ms_per_step": ms_plain,
                  "calls_per_step": len(arrays), "speedup_batched_over_plain": ms_plain / ms_batched},
        "per_kernel_ms": {k: t for k, (l, t) in prof.items()},
        "gpu_launches": int(sum(l for l, _ in prof.values())),
        "e2e": {"value": rows / (e2e_ms / 1e3), "unit": "rows/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(4 * rows)},
        "tile_shapes": am.batch_tuning(),
        "clocks": clocks.summary(),
    }
    if emit:
        print(json.dumps(line))
    return line


SERVE_TABLE_ROWS = 50_000_000


def make_serving_tables(am, rows=SERVE_TABLE_ROWS, seed=SEED + 3):
    """The served stream's resident tables: an int64 key over the whole range (as the single-key case),
    a float64 key ~ N(0, 1), and an (int32 uniform, int64 in [0, 2^40) with 10% nulls) key pair; each
    with a float64 ~ N(0, 1) and an int32 payload column."""
    import pyarrow as pa
    rng = np.random.default_rng(seed)

    def payload():
        return {"p1": pa.array(rng.standard_normal(rows)),
                "p2": pa.array(rng.integers(-2**31, 2**31 - 1, rows, dtype=np.int32, endpoint=True))}

    def resident(name, cols):
        return am.PlanSource(name, {k: am.MetalArray.from_arrow(v) for k, v in cols.items()})

    t_int = resident("t_int64", {"k": pa.array(rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, rows,
                                                            dtype=np.int64, endpoint=True)), **payload()})
    t_f64 = resident("t_float64", {"k": pa.array(rng.standard_normal(rows)), **payload()})
    k2 = rng.integers(0, 2**40, rows, dtype=np.int64)
    t_two = resident("t_pair", {"k1": pa.array(rng.integers(-2**31, 2**31 - 1, rows, dtype=np.int32, endpoint=True)),
                                "k2": pa.array(k2, mask=rng.random(rows) < 0.10), **payload()})
    return [(t_int, ["k"]), (t_f64, ["k"]), (t_two, ["k1", "k2"])]


def serving_requests(count, rows=SERVE_TABLE_ROWS, seed=SEED + 5):
    """Request i: (table index, offset, length); lengths log-uniform in [1e4, 5e7]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(round(10 ** rng.uniform(4, np.log10(5e7))))
        out.append((int(rng.integers(3)), int(rng.integers(0, rows - n + 1)), n))
    return out


def run_serving(args, am, torch, local, emit=True):
    """The served stream: open-loop Poisson arrivals at --rate requests/s against resident tables for
    --serve-seconds, each request sorting a slice by its table's key(s) and taking the 2 payload columns;
    admission cap 120 GB. Reports p50/p99 latency (submission to completion) and rows/s; then the same
    kind of requests all at once through the server against one thread running them back to back
    through am_plan_run (the plain per-call path)."""
    import threading as th
    tables = make_serving_tables(am)
    am.synchronize()
    rate = args.rate
    count = int(rate * args.serve_seconds)
    reqs = serving_requests(count)
    gaps = np.random.default_rng(SEED + 6).exponential(1.0 / rate, count)
    arrivals = np.cumsum(gaps)

    def submit(srv, r):
        t, off, n = r
        src, keys = tables[t]
        return srv.submit(src, off, n, keys, ["p1", "p2"])

    lat = []
    with ClockSampler(local) as clocks, am.Server(workers=4, hbm_cap_bytes=120 * 10**9, batch_rows=1 << 20) as srv:
        tickets = []
        done = th.Event()

        def collect():
            for i in range(count):
                while i >= len(tickets):
                    time.sleep(0.0005)
                _, ms = srv.wait(tickets[i])
                lat.append(ms)
            done.set()

        c = th.Thread(target=collect)
        c.start()
        t0 = time.perf_counter()
        for i, r in enumerate(reqs):
            delay = arrivals[i] - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            tickets.append(submit(srv, r))
        c.join()
        wall = time.perf_counter() - t0
        open_stats = srv.stats()
    served_rows = sum(r[2] for r in reqs)
    by_size = {}
    sizes = np.array([r[2] for r in reqs])
    tabs = np.array([r[0] for r in reqs])
    latv = np.array(lat)
    for lo in (1e4, 1e5, 1e6, 1e7):
        m = (sizes >= lo) & (sizes < lo * 10)
        if m.any():
            by_size[f"{int(lo):.0e}"] = {"count": int(m.sum()), "p50_ms": float(np.percentile(latv[m], 50)),
                                         "p99_ms": float(np.percentile(latv[m], 99)), "max_ms": float(latv[m].max()),
                                         "by_table_max_ms": [float(latv[m & (tabs == t)].max()) if (m & (tabs == t)).any()
                                                             else None for t in range(3)]}
    slow = np.argsort(latv)[-8:]
    slowest = [{"i": int(i), "table": int(tabs[i]), "rows": int(sizes[i]), "ms": float(latv[i]),
                "arrival_s": float(arrivals[i])} for i in slow]

    # Saturation: the same distribution, all requests at once, against the plain per-call path. Each
    # form runs the whole set SAT_REPS times and keeps its best time (the same rule for all three).
    sat = serving_requests(args.sat_requests, seed=SEED + 7)
    sat_rows = sum(r[2] for r in sat)
    with am.Server(workers=4, hbm_cap_bytes=120 * 10**9, batch_rows=1 << 20) as srv:
        for r in sat[:8]:                       # warm-up
            srv.wait(submit(srv, r))
        torch.cuda.synchronize()
        served_s = float("inf")
        for _ in range(SAT_REPS):
            t0 = time.perf_counter()
            ts = [submit(srv, r) for r in sat]
            for t in ts:
                srv.wait(t)
            served_s = min(served_s, time.perf_counter() - t0)
        sat_stats = srv.stats()
    # The same saturation with shared sorts turned off: continuous batching of the small requests and
    # overlap on the device only.
    os.environ["ARROWMETAL_SERVER_SHARED"] = "0"
    try:
        with am.Server(workers=4, hbm_cap_bytes=120 * 10**9, batch_rows=1 << 20) as srv:
            for r in sat[:8]:
                srv.wait(submit(srv, r))
            torch.cuda.synchronize()
            unshared_s = float("inf")
            for _ in range(SAT_REPS):
                t0 = time.perf_counter()
                ts = [submit(srv, r) for r in sat]
                for t in ts:
                    srv.wait(t)
                unshared_s = min(unshared_s, time.perf_counter() - t0)
    finally:
        os.environ.pop("ARROWMETAL_SERVER_SHARED", None)
    for r in sat[:8]:
        t, off, n = r
        plain_run(am, tables[t], off, n)
    am.synchronize()
    plain_s = float("inf")
    for _ in range(SAT_REPS):
        t0 = time.perf_counter()
        for t, off, n in sat:
            plain_run(am, tables[t], off, n)
        am.synchronize()
        plain_s = min(plain_s, time.perf_counter() - t0)

    line = {
        "metric": METRIC, "value": sat_rows / served_s, "unit": "rows/s", "n_gpus": 1,
        "steps": args.sat_requests, "warmup": 8, "ms_per_step": 1e3 * served_s / args.sat_requests,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64/float64/int32",
        "data": "synthetic",
        "config": {"workload": "served sort stream: resident 50M-row tables (int64, float64, (int32, int64) keys, "
                               "2 payload columns), requests of log-uniform 1e4-5e7 rows sorting a slice and "
                               "taking both payloads, HBM admission cap 120 GB, 4 worker streams, batches of "
                               "single-key requests up to 2^20 rows, queued requests of one table and key "
                               "sharing one sort of the rows they cover",
                   "rate_req_s": rate, "requests": count, "saturation_requests": args.sat_requests},
        "open_loop": {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                      "mean_ms": float(np.mean(lat)), "rows_per_s": served_rows / wall, "seconds": wall,
                      "by_size": by_size, "slowest": slowest, "server": open_stats},
        "saturation": {"served_rows_per_s": sat_rows / served_s, "plain_rows_per_s": sat_rows / plain_s,
                       "speedup_served_over_plain": plain_s / served_s, "rows": sat_rows, "server": sat_stats,
                       "without_shared_sorts": {"served_rows_per_s": sat_rows / unshared_s,
                                                "speedup_served_over_plain": plain_s / unshared_s}},
        "clocks": clocks.summary(),
    }
    del tables
    if emit:
        print(json.dumps(line))
    return line


def run_single(args, am, torch, stream, local, workload=None, emit=True):
    """--workload full_range: argsort of 1,000,000 int64 keys over the whole range, uint64 indices
    (am_argsort_ex3, index width 8); --workload multikey: the 50M-row two-key sort (key1 int32 Zipf
    descending, key2 float64 with specials and nulls ascending) and the take of its float64 payload."""
    import pyarrow as pa
    workload = workload or args.workload
    if workload == "full_range":
        arr = pa.array(make_full_range_keys(1_000_000))
        src = am.MetalArray.from_arrow(arr)
        rows = len(arr)

        def step():
            out = src.argsort64()
            del out
        description = "argsort of 1,000,000 int64 keys uniform over the whole int64 range, no nulls, uint64 indices"
        h2d, d2h = arr.nbytes, 8 * rows
        e2e_fn = lambda: am.MetalArray.from_arrow(arr).argsort64().to_arrow()
        dtype = "int64"
    else:
        key1, key2, valid2, payload = make_multikey_table(N_ROWS)
        a1, a2 = pa.array(key1), pa.array(key2, mask=~valid2, from_pandas=False)
        ap = pa.array(payload)
        d1, d2, dp = (am.MetalArray.from_arrow(x) for x in (a1, a2, ap))
        rows = N_ROWS

        def step():
            idx = am.lexsort_indices([d1, d2], descending=[True, False], null_placement="at_end", float_order="ieee")
            out = am.take_columns([d1, d2, dp], idx)
            del idx, out
        description = ("ORDER BY key1 DESC (int32, 200 distinct values, Zipf 1.1), key2 ASC (float64 N(0,1e6) with "
                    "-0.0/+0.0/+inf/-inf 0.5% each, 1% NaN, 5% nulls), nulls last, ieee order; take of the 2 keys "
                    "and a float64 payload; 50,000,000 rows")
        h2d = a1.nbytes + a2.nbytes + ap.nbytes
        d2h = 4 * rows + 8 * rows + rows // 8 + 8 * rows

        def e2e_fn():
            h = [am.MetalArray.from_arrow(x) for x in (a1, a2, ap)]
            idx = am.lexsort_indices(h[:2], descending=[True, False], null_placement="at_end", float_order="ieee")
            return [o.to_arrow() for o in am.take_columns(h, idx)]
        dtype = "int32/float64"
    for _ in range(max(args.warmup, 3)):
        step()
    am.synchronize()
    steps = max(3, min(args.steps, 100))
    am.profile(True)
    am.profile_reset()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(steps):
            step()
        ev1.record(stream)
        ev1.synchronize()
        am.synchronize()
    ms_profiled = ev0.elapsed_time(ev1) / steps
    prof = am.profile_entries()
    am.profile(False)
    # The same steps again without the per-launch events: the step time reported.
    am.synchronize()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(steps):
        step()
    ev1.record(stream)
    ev1.synchronize()
    am.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    e2e = []
    for i in range(4):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = e2e_fn()
        e2e.append(time.perf_counter() - t0)
        del r
    e2e_ms = 1e3 * statistics.median(e2e[1:])
    line = {
        "metric": METRIC, "value": rows / (ms / 1e3), "unit": "rows/s", "n_gpus": 1, "steps": steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": dtype, "data": "synthetic", "config": {"workload": description, "rows": rows},
        "ms_per_step_profiled": ms_profiled,
        "per_kernel_ms_per_step": {k: t / steps for k, (l, t) in prof.items()},
        "gpu_launches": int(sum(l for l, _ in prof.values())),
        "e2e": {"value": rows / (e2e_ms / 1e3), "unit": "rows/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "clocks": clocks.summary()}
    if emit:
        print(json.dumps(line))
    return line


def run_topk(args, am, torch, stream, local):
    """--workload topk: ORDER BY key LIMIT k on the 50M-row key column (int64 in [0, 2^40), 10% nulls):
    am_top_k_ex (radix selection) for several k against the full argsort, CUDA events per call."""
    import pyarrow as pa
    key, valid, _, _ = make_table(N_ROWS)
    col = am.MetalArray.from_arrow(pa.array(key, mask=~valid))

    def timed(fn, reps):
        for _ in range(3):
            fn()
        am.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(reps):
            fn()
        ev1.record(stream)
        ev1.synchronize()
        am.synchronize()
        return ev0.elapsed_time(ev1) / reps

    with ClockSampler(local) as clocks:
        full_ms = timed(lambda: col.argsort(False, "at_end"), 20)
        per_k = {str(k): timed(lambda: col.top_k(k, False, "at_end"), 20) for k in (10, 1000, 100_000, 1_000_000)}
    k_head = "1000"
    print(json.dumps({
        "metric": METRIC, "value": N_ROWS / (per_k[k_head] / 1e3), "unit": "rows/s", "n_gpus": 1, "steps": 20,
        "warmup": 3, "ms_per_step": per_k[k_head], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int64", "data": "synthetic",
        "config": {"workload": "ORDER BY key LIMIT 1000 (am_top_k_ex) on 50,000,000 int64 keys in [0, 2^40) with "
                               "10% nulls, uint32 indices", "rows": N_ROWS},
        "top_k_ms": per_k, "full_argsort_ms": full_ms, "clocks": clocks.summary()}))


def run_consumers(args, am, torch, stream, local):
    """--workload consumers: the sort consumers on the 50M-row key column (int64 in [0, 2^40), 10% nulls)
    and on a 50M-row low-cardinality column (1,000 distinct int64 values, 10% nulls): partition_nth_indices
    at the median, rank, rank_quantile, row_number, unique and value_counts, against the full argsort;
    CUDA events per call."""
    import pyarrow as pa
    key, valid, _, _ = make_table(N_ROWS)
    col = am.MetalArray.from_arrow(pa.array(key, mask=~valid))
    rng = np.random.default_rng(SEED + 9)
    low = am.MetalArray.from_arrow(pa.array(rng.integers(0, 1000, N_ROWS, dtype=np.int64),
                                            mask=rng.random(N_ROWS) < 0.10))

    def timed(fn, reps):
        for _ in range(3):
            fn()
        am.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(reps):
            fn()
        ev1.record(stream)
        ev1.synchronize()
        am.synchronize()
        return ev0.elapsed_time(ev1) / reps

    reps = max(args.steps, 3)
    with ClockSampler(local) as clocks:
        ms = {
            "argsort": timed(lambda: col.argsort(False, "at_end"), reps),
            "partition_nth_median": timed(lambda: col.partition_nth_indices(N_ROWS // 2), reps),
            "rank_min": timed(lambda: col.rank(), reps),
            "rank_dense_low_cardinality": timed(lambda: low.rank(tiebreaker="dense"), reps),
            "rank_quantile": timed(lambda: col.rank_quantile(), reps),
            "row_number": timed(lambda: col.row_number(), reps),
            "unique_sorted": timed(lambda: col.unique("sorted"), reps),
            "value_counts_low_cardinality": timed(lambda: low.value_counts(), reps),
        }
    head = ms["partition_nth_median"]
    print(json.dumps({
        "metric": METRIC, "value": N_ROWS / (head / 1e3), "unit": "rows/s", "n_gpus": 1, "steps": reps,
        "warmup": 3, "ms_per_step": head, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int64", "data": "synthetic",
        "config": {"workload": "partition_nth_indices at the median (am_partition_nth_ex) on 50,000,000 int64 keys "
                               "in [0, 2^40) with 10% nulls, uint32 indices; the other sort consumers beside it",
                   "rows": N_ROWS},
        "consumer_ms": ms, "clocks": clocks.summary()}))


def run_external(args, am, torch, local):
    """--workload external: the out-of-core sort of a record-batch stream (am_stream_sort_ex) over
    100,000,000 rows in host memory (int64 key in [0, 2^40) with 10% nulls, float64 and int32 payload;
    1M-row batches), collected back into host memory: once as one run in HBM, once with a 256 MiB run
    budget, which spills 8+ sorted runs to the scratch directory and merges them on the GPU."""
    import pyarrow as pa
    n = 100_000_000
    key, valid, p1, p2 = make_table(n, seed=SEED + 10)
    table = pa.table({"key": pa.array(key, mask=~valid), "p1": pa.array(p1), "p2": pa.array(p2)})
    batches = table.to_batches(max_chunksize=1_000_000)
    res = {}
    with ClockSampler(local) as clocks:
        for name, budget in (("in_hbm", None), ("spilled_256MiB_runs", 256 << 20)):
            if budget:
                os.environ["ARROWMETAL_STREAM_RUN_BYTES"] = str(budget)
            try:
                with tempfile.TemporaryDirectory() as scratch:
                    t0 = time.perf_counter()
                    s = am.scan_arrow(pa.RecordBatchReader.from_batches(table.schema, batches))
                    out = s.sort("key", scratch=scratch)
                    wall = time.perf_counter() - t0
            finally:
                os.environ.pop("ARROWMETAL_STREAM_RUN_BYTES", None)
            assert out.num_rows == n
            res[name] = {"wall_s": wall, "rows_per_s": n / wall,
                         **{k: s.stats[k] for k in ("read_s", "gpu_s", "merge_s", "bytes_read")}}
            del out
    head = res["in_hbm"]
    print(json.dumps({
        "metric": METRIC, "value": head["rows_per_s"], "unit": "rows/s", "n_gpus": 1, "steps": 1, "warmup": 0,
        "ms_per_step": head["wall_s"] * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int64", "data": "synthetic",
        "config": {"workload": "external sort of a 100,000,000-row record-batch stream from host memory "
                               "(am_stream_sort_ex, int64 key with 10% nulls + float64 + int32), collected to host",
                   "rows": n, "batch_rows": 1_000_000},
        "external": res, "clocks": clocks.summary()}))


def make_strings(n, seed=SEED + 8):
    """n utf8 strings of 0-24 lowercase letters (uniform length), 5% nulls, built from numpy buffers."""
    import pyarrow as pa
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 25, n).astype(np.int32)
    offs = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(lens, out=offs[1:])
    data = rng.integers(ord("a"), ord("z") + 1, int(offs[-1]), dtype=np.uint8)
    valid = rng.random(n) >= 0.05
    return pa.Array.from_buffers(pa.utf8(), n, [pa.py_buffer(np.packbits(valid, bitorder="little")),
                                                pa.py_buffer(offs), pa.py_buffer(data)], null_count=-1)


def run_strings(args, am, torch, stream, local):
    """--workload strings: ORDER BY a utf8 key (10M rows, 0-24 lowercase letters, 5% nulls) + take of a
    float64 payload through am_plan_run; pyarrow's sort_indices + take on the host timed beside it."""
    import pyarrow as pa
    import pyarrow.compute as pc
    n = 10_000_000
    key = make_strings(n)
    pay = pa.array(np.random.default_rng(SEED + 9).standard_normal(n))
    src = am.PlanSource("t", {"s": key, "v": pay})
    plan = {"op": "sort", "by": [["s", False, {"nulls": "last"}]], "input": {"op": "scan", "source": "t"}}
    for _ in range(3):
        am.run_plan(plan, [src])
    am.synchronize()
    am.profile(True)
    am.profile_reset()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = max(3, min(args.steps, 20))
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(steps):
            out = am.run_plan(plan, [src])
            del out
        ev1.record(stream)
        ev1.synchronize()
        am.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    prof = am.profile_entries()
    am.profile(False)
    t0 = time.perf_counter()
    idx = pc.sort_indices(pa.table({"s": key}), [("s", "ascending")], null_placement="at_end")
    key.take(idx), pay.take(idx)
    cpu_s = time.perf_counter() - t0
    print(json.dumps({
        "metric": METRIC, "value": n / (ms / 1e3), "unit": "rows/s", "n_gpus": 1, "steps": steps, "warmup": 3,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "utf8",
        "data": "synthetic",
        "config": {"workload": "ORDER BY utf8 key (0-24 lowercase letters, 5% nulls) + take of the key and a float64 "
                               "payload, 10,000,000 rows", "rows": n},
        "per_kernel_ms_per_step": {k: t / steps for k, (l, t) in prof.items()},
        "cpu_baseline": {"value": n / cpu_s, "unit": "rows/s", "cores": 1, "kind": "pyarrow",
                         "sample": "pyarrow sort_indices + take of the same 10M rows, once"},
        "clocks": clocks.summary()}))


def run_sizes(args, am, torch, stream, local):
    """--workload sizes: the ORDER BY (select_all(sort(scan))) of tables of 1M to 50M rows, for the
    benchmark's key (int64 in [0, 2^40), 10% nulls) and for full-range int64 keys, each with the float64
    and int32 payload columns; CUDA events, median of the steps. For choosing size thresholds."""
    import pyarrow as pa
    res = {}
    rng = np.random.default_rng(SEED + 11)
    for n in (1 << 20, 1 << 21, 1 << 22, 1 << 23, 1 << 24, 1 << 25, 40_000_000, N_ROWS):
        p1 = pa.array(rng.standard_normal(n))
        p2 = pa.array(rng.integers(-2**31, 2**31 - 1, n, dtype=np.int32, endpoint=True))
        for kind in ("bench_key", "full_range"):
            if kind == "bench_key":
                key = pa.array(rng.integers(0, 2**40, n, dtype=np.int64), mask=rng.random(n) < 0.10)
            else:
                key = pa.array(rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, n, dtype=np.int64,
                                            endpoint=True))
            src = am.PlanSource("t", {"c0": key, "c1": p1, "c2": p2})
            for _ in range(3):
                am.run_plan(PLAN, [src])
            am.synchronize()
            st = am.last_sort_stats()
            times = []
            for _ in range(max(5, min(args.steps, 20))):
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                ev0.record(stream)
                out = am.run_plan(PLAN, [src])
                ev1.record(stream)
                ev1.synchronize()
                del out
                times.append(ev0.elapsed_time(ev1))
            ms = statistics.median(times)
            res[f"{kind}/{n}"] = {"ms": ms, "rows_per_s": n / (ms / 1e3), "passes_run": st["passes_run"],
                                  "records": st["payload_in_records"]}
            del src
    print(json.dumps({"metric": METRIC, "workload": "sizes", "unit": "ms",
                      "hybrid_min_rows": os.environ.get("ARROWMETAL_HYBRID_MIN_ROWS", "default"), "sizes": res}))


def plain_run(am, table, offset, n):
    """One request through am_plan_run on the calling thread (the plain per-call path)."""
    src, keys = table
    cols = list(keys) + ["p1", "p2"]
    sel = [[c, f'(col "{c}")'] for c in cols]
    plan = {"op": "select", "exprs": sel, "input": {"op": "sort", "by": [[k, False, {"nulls": "last"}] for k in keys],
            "input": {"op": "select", "exprs": sel, "input": {"op": "limit", "count": n, "offset": offset,
                                                                "input": {"op": "scan", "source": src.name}}}}}
    out = am.run_plan(plan, [src])
    del out


def arrow_columns(key, valid, p1, p2):
    import pyarrow as pa
    return {"c0": pa.array(key, mask=~valid), "c1": pa.array(p1), "c2": pa.array(p2)}


PLAN = json.dumps({"op": "select", "exprs": [[f"c{i}", f'(col "c{i}")'] for i in range(3)],
                   "input": {"op": "sort", "by": [["c0", False, {"nulls": "last"}]],
                             "input": {"op": "scan", "source": "t"}}})


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        if not self.proc or not self.path:
            return None
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def algorithmic_bytes(n, m, passes, local_sort=False, records=False):
    """Bytes each kernel of one step must move once (the roofline's model, per step):
    - histogram: reads the key column (8 B a row) and its validity bitmap;
    - digit passes: the first reads the key column and bitmap again and writes the m value rows'
      (key, id) and the n - m null rows' id and zeroed key straight to their final places; a middle
      pass reads and writes m (key, id); the last reads m (key, id) and writes m ids and m rebuilt key
      values;
    - local sorts (the two-level sort of one large key, after its two passes on the top digits): read
      m (key, id) and write m ids and m rebuilt key values;
    - take: reads the n ids once and gathers and writes the two payload columns (8 + 4 B a row);
    - sort_finish: writes the sorted key column's validity bitmap.
    The bucket-start kernel of the two-level sort moves no compulsory bytes (like the plan).

    With the payload carried in row records (`records`: the table is in HBM), each value row moves a
    16-byte record (id + 12 payload bytes) beside its 8-byte key instead of a 4-byte id, and there is no
    take:
    - first pass: reads the key column, its bitmap and the two payload columns (12 B a row), writes
      each value row's key and record (24 B) and each null row's key value and payload (8 + 12 B);
    - a middle pass reads and writes 24 B a value row;
    - the local sorts (or the last pass) read 24 B a value row and write its key value and payload
      (8 + 12 B)."""
    src = 8 * n + n / 8
    if records:
        first = src + 12 * n + 24 * m + 20 * (n - m)
        last = 24 * m + 20 * m
        if passes <= 1:
            pass_bytes = src + 12 * n + 20 * n
        elif local_sort:
            pass_bytes = first + (passes - 1) * 48 * m
        else:
            pass_bytes = first + (passes - 2) * 48 * m + last
        out = {"radix_histogram": src, "radix_onesweep_pass": pass_bytes, "sort_finish": n / 8}
        if local_sort:
            out["radix_local_sort"] = last
        return out
    if passes <= 1:
        pass_bytes = src + 12 * n
    else:
        first = src + 12 * m + 12 * (n - m)
        pass_bytes = first + (passes - 2) * 24 * m + 24 * m
    out = {"radix_histogram": src, "radix_onesweep_pass": pass_bytes,
           "take_gather": 4 * n + 2 * (8 + 4) * n, "sort_finish": n / 8}
    if local_sort:
        out["radix_local_sort"] = 24 * m
    return out


# DRAM bytes (read + write) per row of the workload, per kernel and step: dram__bytes_read.sum +
# dram__bytes_write.sum of the kernel's launches in one sort, from one ncu capture of this benchmark at
# 25,000,000 rows (22.5M value rows: the two-level sort runs as at 50M), divided by the rows. Keyed by
# whether the payload rode through the sort in records (the table in HBM) or was gathered afterwards.
TRAFFIC_PER_ROW = {
    True: {"radix_histogram": 8.26, "radix_onesweep_pass": 83.97, "radix_local_sort": 38.00},
    False: {},
}


def traffic_per_step(kernel, n, records):
    b = TRAFFIC_PER_ROW[bool(records)].get(kernel)
    return None if b is None else b * n


def cpu_oracle_rate(key, valid, p1, p2, threads):
    """The CPU oracle on the whole workload once: argsort (C restatement, `threads` threads) and the
    take of the 3 columns (C restatement, one thread per column)."""
    import pyarrow as pa
    from oracle import oracle
    cols = arrow_columns(key, valid, p1, p2)
    t0 = time.perf_counter()
    idx = oracle.argsort(cols["c0"], threads=threads)
    ia = pa.array(idx)
    ths = [threading.Thread(target=oracle.take, args=(cols[c], ia)) for c in cols]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    dt = time.perf_counter() - t0
    return len(key) / dt, dt


def pyarrow_rate(key, valid, p1, p2, rows=10_000_000, repeats=3):
    """pyarrow's sort_indices + Table.take (the reference's own oracle for this order) on the first
    `rows` rows of the workload: one warm-up, then the best of `repeats`."""
    import pyarrow as pa
    import pyarrow.compute as pc
    rows = min(rows, len(key))
    t = pa.table(arrow_columns(key[:rows], valid[:rows], p1[:rows], p2[:rows]))
    best = float("inf")
    for i in range(repeats + 1):
        t0 = time.perf_counter()
        idx = pc.sort_indices(t, sort_keys=[("c0", "ascending")], null_placement="at_end")
        out = t.take(idx)
        dt = time.perf_counter() - t0
        del idx, out
        if i > 0:
            best = min(best, dt)
    return {"value": rows / best, "unit": "rows/s", "cores": os.cpu_count() or 1, "pyarrow_cpu_count": pa.cpu_count(),
            "kind": "pyarrow", "version": pa.__version__,
            "sample": f"the first {rows:,} rows of the workload: sort_indices + Table.take of the 3 columns, "
                      f"best of {repeats} after one warm-up ({best:.2f} s)"}


def datafusion_baseline():
    """DataFusion's SortExec on the workload when the datafusion package is importable here."""
    try:
        import datafusion  # noqa: F401
    except ImportError:
        return {"unavailable": "unavailable on this box: the datafusion Python package is not installed and there "
                               "is no network; the reference publishes 1,581.22 ms for this ORDER BY on DataFusion "
                               "alone (Apple M4 Max, 16 cores; datafusion/results/datafusion_sort_warm_2026-09-29.csv:376)"}
    return {"unavailable": "datafusion is importable but not timed by this benchmark"}


def compact(line, drop=("metric", "unit", "n_gpus", "higher_is_better", "scaling", "vs_baseline", "data")):
    """A configuration's line as a sub-object of the headline line (its shared keys dropped)."""
    return {k: v for k, v in line.items() if k not in drop}


def sub_workloads(args, am, torch, stream, local):
    """The single-key scale case, the two-key sort, the segmented batch and the served stream, run after
    the headline (one GPU); each is measured with its own CUDA events and clock record."""
    import copy
    out = {}
    a = copy.copy(args)
    a.steps = min(args.steps, 50)
    a.warmup = max(args.warmup, 3)
    out["full_range"] = compact(run_single(a, am, torch, stream, local, "full_range", emit=False))
    am.synchronize()
    out["multikey"] = compact(run_single(a, am, torch, stream, local, "multikey", emit=False))
    am.synchronize()
    b = compact(run_segmented(a, am, torch, stream, local, emit=False))
    b["ratio_batched_over_plain"] = b["plain"]["speedup_batched_over_plain"]
    out["batched"] = b
    am.synchronize()
    sv = copy.copy(a)
    sv.serve_seconds = min(args.serve_seconds, args.sub_serve_seconds)
    sv.sat_requests = min(args.sat_requests, args.sub_sat_requests)
    s = compact(run_serving(sv, am, torch, local, emit=False))
    s["p50_ms"] = s["open_loop"]["p50_ms"]
    s["p99_ms"] = s["open_loop"]["p99_ms"]
    s["ratio_served_over_plain"] = s["saturation"]["speedup_served_over_plain"]
    s["ratio_served_over_plain_without_shared_sorts"] = \
        s["saturation"]["without_shared_sorts"]["speedup_served_over_plain"]
    out["served"] = s
    return out


def max_over_ranks(x, dist, device):
    """The largest of every rank's `x` (a time): the whole job is as slow as its slowest replica."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(rows_per_rank, world, ms):
    """Rows all replicas processed per second, over the slowest replica's time per step."""
    return world * rows_per_rank / (ms / 1e3)


def run_reference_arm(args, rank):
    """--impl reference: the reference's sort path on the host's cores. The reference is Swift + Metal
    and runs on no machine here, so the C restatement of its algorithm in oracle/ stands in for it."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    # Size each step so that warm-up + timed steps take about two minutes.
    probe = make_table(1_000_000, SEED)
    rate, _ = cpu_oracle_rate(*probe, threads)
    budget = 120.0 / max(1, args.steps + args.warmup)
    n = int(min(args.rows, N_ROWS, max(100_000, rate * budget)))
    key, valid, p1, p2 = make_table(n, SEED)
    for _ in range(args.warmup):
        cpu_oracle_rate(key, valid, p1, p2, threads)
    times = [cpu_oracle_rate(key, valid, p1, p2, threads)[1] for _ in range(args.steps)]
    ms = 1e3 * sum(times) / len(times)
    value = n / (ms / 1e3)
    sample = f"the first {n:,} rows of the workload per step (same generator), argsort + take of 3 columns"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "rows_per_step": n},
        "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--e2e-inflight", type=int, default=2,
                    help="end-to-end steps in flight at once, pipelined in one thread (1: one at a time)")
    ap.add_argument("--rows", type=int, default=N_ROWS)
    ap.add_argument("--impl", default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="order_by",
                    choices=["order_by", "segmented", "serving", "full_range", "multikey", "topk", "strings",
                             "consumers", "external", "sizes"],
                    help="order_by: the 50M-row ORDER BY (the headline); segmented: 2,048 arrays in one call; "
                         "serving: the served request stream; full_range: 1M full-range int64 keys; multikey: "
                         "the 50M-row two-key sort; topk: ORDER BY ... LIMIT k by radix selection; strings: ORDER BY a utf8 key; "
                         "consumers: partition_nth, rank, unique and value_counts on 50M rows; "
                         "external: the out-of-core sort of a 100M-row batch stream")
    ap.add_argument("--rate", type=float, default=200.0, help="serving: requests per second")
    ap.add_argument("--serve-seconds", type=float, default=30.0, help="serving: length of the open-loop stream")
    ap.add_argument("--sat-requests", type=int, default=400, help="serving: requests of the saturation run")
    ap.add_argument("--headline-only", action="store_true",
                    help="the default run: measure only the 50M-row ORDER BY, not the other configurations")
    ap.add_argument("--sub-serve-seconds", type=float, default=10.0,
                    help="the default run's served stream: length of its open-loop part")
    ap.add_argument("--sub-sat-requests", type=int, default=400,
                    help="the default run's served stream: requests of its saturation part")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank)

    os.environ["ARROWMETAL_DEVICE"] = str(local)
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    import pyarrow as pa
    import arrowmetal_b200 as am

    if args.workload == "segmented":
        stream = torch.cuda.Stream()
        am.set_stream(stream.cuda_stream)
        if rank == 0:
            run_segmented(args, am, torch, stream, local)
        return
    if args.workload == "serving":
        if rank == 0:
            run_serving(args, am, torch, local)
        return
    if args.workload == "strings":
        stream = torch.cuda.Stream()
        am.set_stream(stream.cuda_stream)
        if rank == 0:
            run_strings(args, am, torch, stream, local)
        return
    if args.workload == "topk":
        stream = torch.cuda.Stream()
        am.set_stream(stream.cuda_stream)
        if rank == 0:
            run_topk(args, am, torch, stream, local)
        return
    if args.workload == "external":
        if rank == 0:
            run_external(args, am, torch, local)
        return
    if args.workload == "sizes":
        stream = torch.cuda.Stream()
        am.set_stream(stream.cuda_stream)
        if rank == 0:
            run_sizes(args, am, torch, stream, local)
        return
    if args.workload == "consumers":
        stream = torch.cuda.Stream()
        am.set_stream(stream.cuda_stream)
        if rank == 0:
            run_consumers(args, am, torch, stream, local)
        return
    if args.workload in ("full_range", "multikey"):
        stream = torch.cuda.Stream()
        am.set_stream(stream.cuda_stream)
        if rank == 0:
            run_single(args, am, torch, stream, local)
        return

    n = args.rows
    key, valid, p1, p2 = make_table(n, SEED + rank)
    m_rows = int(valid.sum())
    cols = arrow_columns(key, valid, p1, p2)
    stream = torch.cuda.Stream()
    am.set_stream(stream.cuda_stream)

    # ---- device-resident inputs (imported through the C ABI once)
    dcols = {k: am.MetalArray.from_arrow(v) for k, v in cols.items()}
    src = am.PlanSource("t", dcols)

    def step():
        out = am.run_plan(PLAN, [src])
        del out

    for _ in range(max(args.warmup, 3)):
        step()
    am.synchronize()
    # passes run per sort and whether the payload rode in records, for the byte model
    step()
    st = am.last_sort_stats()

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    peak, peak_kind = measured_peak()
    # The timed region: K steps with no per-launch events.
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        barrier()
        am.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        ev1.synchronize()
        am.synchronize()
        barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    ms = max_over_ranks(ms, dist, "cuda")
    value = whole_job_rate(n, world, ms)
    # The per-kernel split, from a second loop with a CUDA event pair around every launch.
    prof_steps = max(3, min(args.steps, 50))
    am.profile(True)
    am.profile_reset()
    ep0, ep1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ep0.record(stream)
    for _ in range(prof_steps):
        step()
    ep1.record(stream)
    ep1.synchronize()
    am.synchronize()
    ms_profiled = ep0.elapsed_time(ep1) / prof_steps
    prof = am.profile_entries()
    am.profile(False)

    # ---- roofline of the dominant kernel (the take's kernels count as one stage: their model bytes
    # are the take's, however the gather is organised)
    # (the two-level sort: two passes, then the local sorts, when its timer ran and the stats count 2)
    model = algorithmic_bytes(n, m_rows, st["passes_run"],
                              local_sort=st["passes_run"] == 2 and "radix_local_sort" in prof,
                              records=st["payload_in_records"])
    stages = {}
    for name, (launches, total_ms) in prof.items():
        stage = "take_gather" if name.startswith("take_") else name
        e = stages.setdefault(stage, {"launches": 0, "total_ms": 0.0, "kernels": {}})
        e["launches"] += launches
        e["total_ms"] += total_ms
        e["kernels"][name] = {"launches": launches, "ms_per_step": total_ms / prof_steps}
    per_kernel = {}
    for stage, e in stages.items():
        if stage in model:
            b = model[stage] * prof_steps
            e.update({"bytes": b, "gbs": b / (e["total_ms"] / 1e3) / 1e9})
        per_kernel[stage] = e
    dom = max((k for k in per_kernel if "gbs" in per_kernel[k]), key=lambda k: per_kernel[k]["total_ms"])
    d = per_kernel[dom]
    gpu_launches = sum(l for l, _ in prof.values()) * args.steps // prof_steps

    # ---- end to end through the C ABI with host buffers: the inputs sit in pinned host memory (copied
    # there once, before timing); every step imports them, runs the plan and exports the result.
    pinned_keep = []

    def pinned_array(arr):
        bufs = []
        for b in arr.buffers():
            if b is None:
                bufs.append(None)
                continue
            t = torch.empty(b.size, dtype=torch.uint8, pin_memory=True)
            t.numpy()[:] = np.frombuffer(b, dtype=np.uint8)
            pinned_keep.append(t)
            bufs.append(pa.py_buffer(t.numpy()))
        return pa.Array.from_buffers(arr.type, len(arr), bufs, null_count=arr.null_count, offset=arr.offset)

    host_cols = {k: pinned_array(v) for k, v in cols.items()}
    h2d = sum(c.nbytes for c in (key, p1, p2)) + (n + 7) // 8
    e2e_times = []
    d2h = 0
    for i in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hc = {k: am.MetalArray.from_arrow(v) for k, v in host_cols.items()}
        s2 = am.PlanSource("t", hc)
        out = am.run_plan(PLAN, [s2])
        res = {k: v.to_arrow() for k, v in out.items()}
        dt = time.perf_counter() - t0
        if i > 0:
            e2e_times.append(dt)
        d2h = sum(sum(b.size for b in r.buffers() if b is not None) for r in res.values())
        del hc, s2, out, res
    e2e_ms = max_over_ranks(1e3 * statistics.median(e2e_times) if e2e_times else float("nan"), dist, "cuda")

    # ---- the same steps pipelined in this thread: step i + 1's imports and plan are enqueued before step
    # i's results are exported, so one step's uploads run while the previous step's results download (the
    # two copy directions). Every step still imports its own inputs from pinned host memory and exports its
    # whole result to host memory; the time is the whole run's, fill and drain included, over its steps.
    inflight_ms = None
    if args.e2e_steps > 0 and args.e2e_inflight > 1:
        depth = args.e2e_inflight
        sets = [host_cols] + [{k: pinned_array(v) for k, v in cols.items()} for _ in range(depth - 1)]

        def pipelined(nsteps):
            queue = []
            t0 = time.perf_counter()
            for i in range(nsteps + depth - 1):
                if i < nsteps:
                    hc = {k: am.MetalArray.from_arrow(v) for k, v in sets[i % depth].items()}
                    queue.append((hc, am.run_plan(PLAN, [am.PlanSource("t", hc)])))
                    del hc
                if len(queue) >= depth or i >= nsteps:
                    hc0, out0 = queue.pop(0)
                    res = {k: v.to_arrow() for k, v in out0.items()}
                    del hc0, out0, res
            return time.perf_counter() - t0

        pipelined(depth + 2)                            # the pool's blocks for `depth` steps at once
        pipe_steps = max(args.e2e_steps, 4 * depth)
        inflight_ms = max_over_ranks(1e3 * pipelined(pipe_steps) / pipe_steps, dist, "cuda")
        del sets

    line = {
        "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "rows": n, "value_rows": m_rows, "radix_passes_run": st["passes_run"],
                   "radix_passes_skipped": st["passes_skipped"], "parallelism": f"replicas x{world}",
                   "payload": "carried through the sort in row records" if st["payload_in_records"]
                              else "gathered through the permutation after the sort",
                   "l2": "inputs larger than L2 (400 MB key column), no flush"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": d["gbs"], "peak": peak, "unit": "GB/s",
                     "frac": d["gbs"] / peak, "peak_source": peak_kind,
                     "traffic": traffic_per_step(dom, n, st["payload_in_records"]),
                     "per": "one step (all launches of the kernel in one sort)",
                     "pipeline": {"bytes": sum(model.values()), "gbs": sum(model.values()) / (ms / 1e3) / 1e9,
                                  "frac": sum(model.values()) / (ms / 1e3) / 1e9 / peak},
                     "per_kernel": per_kernel},
        "e2e": ({"value": whole_job_rate(n, world, inflight_ms), "unit": "rows/s", "ms_per_step": inflight_ms,
                 "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                 "steps_in_flight": args.e2e_inflight,
                 "one_in_flight": {"value": whole_job_rate(n, world, e2e_ms), "ms_per_step": e2e_ms}}
                if inflight_ms else
                {"value": whole_job_rate(n, world, e2e_ms), "unit": "rows/s", "ms_per_step": e2e_ms,
                 "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps_in_flight": 1}),
        "gpu_launches": int(gpu_launches),
        "clocks": clocks.summary(),
    }
    del src, dcols, host_cols, pinned_keep
    am.synchronize()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, dt = cpu_oracle_rate(key, valid, p1, p2, threads)
        line["cpu_baseline"] = {"value": rate, "unit": "rows/s", "cores": threads, "kind": "port",
                                "sample": f"the whole {n:,}-row workload once ({dt:.2f} s): C oracle argsort on "
                                          f"{threads} threads + take of the 3 columns"}
        line["cpu_baseline_pyarrow"] = pyarrow_rate(key, valid, p1, p2)
        line["cpu_baseline_datafusion"] = datafusion_baseline()
    if rank == 0 and world == 1 and not args.headline_only:
        # The other configurations of the benchmark, each measured in this run with its own clocks.
        line.update(sub_workloads(args, am, torch, stream, local))
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
