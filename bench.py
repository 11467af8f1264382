"""Benchmark of the B200 relational hot path: hash groupby aggregation,
200M rows (Zipf(1.1) int64 keys over 10M distinct values; float64 N(0,1) with
10% nulls; int32 U[0, 1e6)); SUM and MEAN of the float64 column, COUNT(*) and
COUNT of the float64 column, MIN/MAX and NUNIQUE of the int32 column.

`--workload join` / `--workload strings` / `--workload sort` instead print one
line per op of the 200M x 20M int32-key joins / the 100M-row string-key
groupby, stable sort and hash partition / a 100M-row int64-key sort (device
ms, rows/s, per-kernel ms).

One step = one groupby_aggregation call through the public API (C ABI) on
device-resident inputs (4.2 GB, far larger than the 126 MB L2, so no flush is
needed).  Prints ONE JSON line (rank 0).  At N=1 the line also carries
`served`: the batched/served mix (8,192 small joins and groupbys arriving at
2,000 req/s) through the continuous-batching server and, for comparison, the
same requests issued one op per launch (--no-served skips it).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU runs (torchrun) are independent replicas: the path is a single-GPU
task body and shards by rows with no data-path collective (weak scaling);
the process group only carries the barrier and the max-over-ranks time.
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "legate-dataframe_b200"))

METRIC = "join/groupby rows/s + % HBM roofline (1 B200); batched p50/p99 vs unbatched"
N_ROWS = 200_000_000
N_KEYS = 10_000_000
AGGS = [
    ("v", "sum", "sum_v"),
    ("v", "mean", "mean_v"),
    (None, "count_all", "count"),
    ("v", "count", "count_v"),
    ("i", "min", "min_i"),
    ("i", "max", "max_i"),
    ("i", "count_distinct", "nunique_i"),
]
IN_BYTES_PER_ROW = 8 + 8 + 1 + 4  # key + f64 + its null mask + i32 (legate layout)


def measured_peak_gbs():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# synthetic input (seeded, generated on the device)
# ---------------------------------------------------------------------------
def make_input_device(n_rows: int, device):
    import torch

    g = torch.Generator(device=device)
    ranks = torch.arange(1, N_KEYS + 1, device=device, dtype=torch.float64)
    w = ranks.pow(-1.1)
    cdf = torch.cumsum(w, 0)
    cdf /= cdf[-1].clone()
    g.manual_seed(3)
    perm = torch.randperm(N_KEYS, device=device, generator=g)
    key_values = perm.to(torch.int64) * 2_654_435_761 + 12_345  # 10M distinct int64 values
    keys = torch.empty(n_rows, dtype=torch.int64, device=device)
    g.manual_seed(1)
    chunk = 50_000_000
    for s in range(0, n_rows, chunk):
        e = min(n_rows, s + chunk)
        u = torch.rand(e - s, dtype=torch.float64, device=device, generator=g)
        r = torch.searchsorted(cdf, u).clamp_(max=N_KEYS - 1)
        keys[s:e] = key_values[r]
        del u, r
    del cdf, w, ranks, perm
    g.manual_seed(4)
    v = torch.randn(n_rows, dtype=torch.float64, device=device, generator=g)
    valid = (torch.rand(n_rows, device=device, generator=g) >= 0.10).to(torch.uint8)
    g.manual_seed(5)
    i = torch.randint(0, 1_000_000, (n_rows,), dtype=torch.int32, device=device, generator=g)
    torch.cuda.synchronize(device)
    return keys, v, valid, i


def device_table(keys, v, valid, i):
    import pyarrow as pa

    from legate_dataframe import LogicalColumn, LogicalTable

    cols = [
        LogicalColumn.from_torch(keys, pa.int64()),
        LogicalColumn.from_torch(v, pa.float64(), valid),
        LogicalColumn.from_torch(i, pa.int32()),
    ]
    return LogicalTable(cols, ["k", "v", "i"])


def host_sample(keys, v, valid, i, n):
    import numpy as np
    import pyarrow as pa

    k = keys[:n].cpu().numpy()
    vv = v[:n].cpu().numpy()
    m = valid[:n].cpu().numpy().astype(bool)
    ii = i[:n].cpu().numpy()
    return pa.table({"k": k, "v": pa.array(vv, mask=~m), "i": ii})


def output_bytes(tbl) -> int:
    total = 0
    for c in tbl.get_columns():
        from legate_dataframe import _native as N

        total += c.size * N.TYPE_WIDTH[c.ldf_type] + (c.size if c.valid is not None else 0)
    return total


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "50", "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for r in rows for j in range(4) if r[5 + j].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def max_over_ranks(value: float, world: int, device) -> float:
    """Max of a per-rank time over all ranks (the slowest replica times the job)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# CPU baselines: the reference's CPU path (Arrow Acero aggregate, the calls of
# GroupByAggregationTask::cpu_variant) on a bounded sample
# ---------------------------------------------------------------------------
def cpu_groupby_rate(sample, use_threads: bool, min_seconds: float = 10.0):
    from oracle import arrow_ref

    t0 = time.perf_counter()
    reps = 0
    while True:
        arrow_ref.groupby(sample, ["k"], AGGS, use_threads=use_threads)
        reps += 1
        el = time.perf_counter() - t0
        if el >= min_seconds or reps >= 20:
            break
    return sample.num_rows * reps / el, el, reps


def run_reference(args):
    """--impl reference: the reference's CPU implementation of the path (Arrow
    Acero aggregate) with every host thread, on bounded samples."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import numpy as np
    import pyarrow as pa

    n = args.ref_rows
    rng = np.random.default_rng(3)
    ranks = np.arange(1, N_KEYS + 1, dtype=np.float64)
    cdf = np.cumsum(ranks ** -1.1)
    cdf /= cdf[-1]
    key_values = rng.permutation(N_KEYS).astype(np.int64) * 2_654_435_761 + 12_345
    k = key_values[np.minimum(np.searchsorted(cdf, np.random.default_rng(1).random(n)), N_KEYS - 1)]
    r4 = np.random.default_rng(4)
    v = r4.normal(size=n)
    m = r4.random(n) < 0.10
    i = np.random.default_rng(5).integers(0, 1_000_000, n).astype(np.int32)
    sample = pa.table({"k": k, "v": pa.array(v, mask=m), "i": i})
    from oracle import arrow_ref

    for _ in range(args.warmup):
        arrow_ref.groupby(sample, ["k"], AGGS, use_threads=True)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        arrow_ref.groupby(sample, ["k"], AGGS, use_threads=True)
    el = time.perf_counter() - t0
    rate = n * args.steps / el
    cores = os.cpu_count()
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "rows/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+int64",
        "data": "synthetic (seeded, config-1 distributions)",
        "config": {"workload": "groupby config 1 (Zipf 1.1 int64 keys over 10M, f64 N(0,1) 10% nulls, i32)",
                   "rows_per_step": n, "full_rows": N_ROWS},
        "cpu_baseline": {"value": rate, "unit": "rows/s", "cores": cores, "kind": "port",
                         "sample": f"{n} rows/step of the config-1 distribution; Arrow {pa.__version__} Acero "
                                   "aggregate (hash_sum/mean/count_all/count/min/max/count_distinct), "
                                   "use_threads=True: the Arrow calls of the reference's cpu_variant"},
        "e2e": {"value": rate, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# served mix: many small joins/groupbys, batched vs one op per launch
# ---------------------------------------------------------------------------
SERVED_CANDIDATES = [(16384, 4, 0.5), (16384, 8, 0.5), (16384, 16, 0.5), (65536, 8, 0.5), (16384, 8, 0.35)]


def run_served(device, n_requests: int):
    """8,192 requests, Poisson arrivals at 2,000 req/s, each an int64-key inner
    join or groupby SUM/COUNT over LogNormal(median 50K, sigma 1) rows clipped
    to 1K-20M, keys uniform over 0.1 x rows; tables resident on the device.
    Reports the continuous-batching server (autotuned) and the same requests
    issued one op per launch, each at the arrival rate (latency) and with all
    requests queued at t=0 (throughput)."""
    from legate_dataframe import _native as N
    from legate_dataframe import serving as S

    reqs = S.make_trace(n_requests=n_requests, seed=12, device=device)
    calib = S.make_trace(n_requests=512, seed=13, device=device)
    best = S.Autotuner().tune(calib, f"served-mix-{n_requests}", arena_bytes=16 << 30, candidates=SERVED_CANDIDATES)
    srv = S.Server(arena_bytes=16 << 30, tile_rows=best["tile_rows"], ctas_per_sm=best["ctas_per_sm"],
                   load_factor=best["load_factor"])
    srv.serve(calib, realtime=False)  # warm-up
    l0 = N.launch_count()
    rt = srv.serve(reqs, realtime=True).summary()
    rt["gpu_launches"] = N.launch_count() - l0
    sat = srv.serve(reqs, realtime=False).summary()
    srv.close()
    S.run_one_op_per_launch(calib[:32], realtime=False)  # warm-up
    l0 = N.launch_count()
    base_rt = S.run_one_op_per_launch(reqs, realtime=True).summary()
    base_rt["gpu_launches"] = N.launch_count() - l0
    base_sat = S.run_one_op_per_launch(reqs, realtime=False).summary()
    rows = sum(q.rows for q in reqs)
    return {
        "workload": f"{n_requests} requests, Poisson 2000 req/s, 50% int64-key inner join / 50% int64-key groupby "
                    "SUM+COUNT(f64, 10% nulls), rows LogNormal(median 50K, sigma 1) clipped 1K-20M, keys U[0, "
                    "0.1 x rows); device-resident tables; latency = arrival -> result on the host",
        "rows": rows,
        "autotune": best,
        "batched": rt,
        "batched_saturated": sat,
        "one_op_per_launch": base_rt,
        "one_op_per_launch_saturated": base_sat,
        "saturated_throughput_ratio": sat["req_per_s"] / base_sat["req_per_s"],
    }


# ---------------------------------------------------------------------------
# other workloads of the path (not the default line): `--workload join` runs
# the 200M x 20M int32-key hash joins, `--workload strings` the 100M-row
# string-key groupby / stable sort / hash partition; one JSON line per op
# with device ms, rows/s and per-kernel ms (CUDA events on the stream)
# ---------------------------------------------------------------------------
def _profiled(N, fn, steps):
    import torch

    for _ in range(2):
        r = fn()
        del r
    torch.cuda.synchronize()
    N.profile_enable(True)
    N.profile_report(reset=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        r = fn()
        rows = r[0].num_rows() if isinstance(r, tuple) else r.num_rows()
        del r
    e1.record()
    torch.cuda.synchronize()
    prof = N.profile_report(reset=True)
    N.profile_enable(False)
    return e0.elapsed_time(e1) / steps, rows, {k: [c // steps, round(t / steps, 3)] for k, (c, t) in
                                               sorted(prof.items(), key=lambda kv: -kv[1][1])}


def run_join_workload(args):
    """Build 20M rows (int32 keys = a permutation of [0, 20M), two int64
    payloads); probe rows (--rows, default 200M): with p=0.8 a build key of
    Zipf(0.9) rank, else U[20M, 40M); 5% null keys; one float64 payload."""
    import pyarrow as pa
    import torch

    from legate_dataframe import LogicalColumn, LogicalTable
    from legate_dataframe import _native as N
    from legate_dataframe.lib.join import JoinType, join

    dev = torch.device("cuda", 0)
    nb, npr = 20_000_000, args.rows
    g = torch.Generator(device=dev)
    g.manual_seed(6)
    bkey = torch.randperm(nb, device=dev, generator=g).to(torch.int32)
    bp1 = torch.randint(-(2**40), 2**40, (nb,), device=dev, generator=g)
    bp2 = torch.randint(-(2**40), 2**40, (nb,), device=dev, generator=g)
    g.manual_seed(7)
    cdf = torch.cumsum(torch.arange(1, nb + 1, device=dev, dtype=torch.float64).pow(-0.9), 0)
    cdf /= cdf[-1].clone()
    u = torch.rand(npr, device=dev, generator=g, dtype=torch.float64)
    hit = torch.rand(npr, device=dev, generator=g) < 0.8
    idx = torch.searchsorted(cdf, u).clamp_(max=nb - 1)
    miss = torch.randint(nb, 2 * nb, (npr,), device=dev, generator=g, dtype=torch.int32)
    pkey = torch.where(hit, bkey[idx], miss)
    pvalid = torch.rand(npr, device=dev, generator=g) >= 0.05
    ppay = torch.rand(npr, device=dev, generator=g, dtype=torch.float64)
    del cdf, u, hit, idx, miss
    lt = LogicalTable([LogicalColumn.from_torch(pkey, pa.int32(), valid=pvalid),
                       LogicalColumn.from_torch(ppay, pa.float64())], ["lk", "lv"])
    rt = LogicalTable([LogicalColumn.from_torch(bkey, pa.int32()), LogicalColumn.from_torch(bp1, pa.int64()),
                       LogicalColumn.from_torch(bp2, pa.int64())], ["rk", "r1", "r2"])
    peak, kind = measured_peak_gbs()
    for jt in (JoinType.INNER, JoinType.LEFT, JoinType.FULL):
        ms, rows, kern = _profiled(N, lambda: join(lt, rt, lhs_keys=["lk"], rhs_keys=["rk"], join_type=jt),
                                   args.steps)
        in_b = nb * 20 + npr * 13
        out_b = rows * (4 + 1 + 8 + 4 + 8 + 8 + (3 if jt != JoinType.INNER else 0))
        print(json.dumps({"workload": f"join {jt.name.lower()}: {npr} probe x {nb} build rows", "ms": round(ms, 3),
                          "rows_per_s": (npr + nb) / (ms / 1e3), "out_rows": rows,
                          "op_GBps_algorithmic": (in_b + out_b) / (ms / 1e3) / 1e9,
                          "op_frac_of_peak": (in_b + out_b) / (ms / 1e3) / 1e9 / peak, "peak_kind": kind,
                          "kernels_ms": kern}), flush=True)
    return 0


def run_strings_workload(args):
    """--rows (default 100M) rows: string key drawn Zipf(1.0) from a 2M-entry
    dictionary of [a-z0-9] strings of length U{8..24}; int64 timestamps over
    one year; float32 LogNormal(0,1) values.  groupby SUM/COUNT(*) on the key,
    stable sort (key asc, ts desc), hash_partition(key, 256)."""
    import numpy as np
    import pyarrow as pa
    import torch

    from legate_dataframe import LogicalColumn, LogicalTable
    from legate_dataframe import _native as N
    from legate_dataframe.lib.groupby_aggregation import groupby_aggregation
    from legate_dataframe.lib.hash_partition import hash_partition
    from legate_dataframe.lib.sort import sort

    dev = torch.device("cuda", 0)
    n, nd = args.rows, 2_000_000
    rng = np.random.default_rng(9)
    lens = rng.integers(8, 25, nd)
    alphabet = np.frombuffer(b"abcdefghijklmnopqrstuvwxyz0123456789", dtype=np.uint8)
    d_chars = torch.from_numpy(alphabet[rng.integers(0, 36, int(lens.sum()))].copy()).to(dev)
    doff = np.zeros(nd + 1, np.int64)
    np.cumsum(lens, out=doff[1:])
    d_off = torch.from_numpy(doff).to(dev)
    g = torch.Generator(device=dev)
    g.manual_seed(9)
    cdf = torch.cumsum(1.0 / torch.arange(1, nd + 1, device=dev, dtype=torch.float64), 0)
    cdf /= cdf[-1].clone()
    pick = torch.searchsorted(cdf, torch.rand(n, device=dev, generator=g, dtype=torch.float64)).clamp_(max=nd - 1)
    row_len = (d_off[1:] - d_off[:-1])[pick]
    row_off = torch.cumsum(row_len, 0) - row_len
    rowid = torch.repeat_interleave(torch.arange(n, device=dev), row_len)
    pos = torch.arange(int(row_len.sum()), device=dev)
    chars = d_chars[d_off[pick][rowid] + (pos - row_off[rowid])]
    del rowid, pos, cdf
    ranges = torch.stack([row_off, row_off + row_len - 1], 1).contiguous()
    t0 = 1_600_000_000_000_000
    ts = torch.randint(t0, t0 + 365 * 86400 * 10**6, (n,), device=dev, generator=g)
    val = torch.exp(torch.randn(n, device=dev, generator=g)).to(torch.float32)
    key = LogicalColumn(pa.string(), N.LDF_STRING, n, ranges.view(torch.uint8).reshape(-1), None, chars=chars,
                        chars_base=0, num_chars=chars.numel())
    t = LogicalTable([key, LogicalColumn.from_torch(ts, pa.timestamp("us")),
                      LogicalColumn.from_torch(val, pa.float32())], ["k", "ts", "v"])
    row_bytes = 16 + chars.numel() / n + 8 + 4
    ops = {
        "groupby SUM/COUNT(*) on the string key": (lambda: groupby_aggregation(
            t, ["k"], [("v", "sum", "s"), (None, "count_all", "c")]), n * (16 + chars.numel() / n + 4)),
        "stable sort (key asc, ts desc)": (lambda: sort(t, ["k", "ts"], sort_ascending=[True, False], stable=True),
                                           2 * n * row_bytes),
        "hash_partition(key, 256)": (lambda: hash_partition(t, ["k"], 256), 2 * n * row_bytes),
    }
    peak, kind = measured_peak_gbs()
    wanted = {"groupby": "groupby", "sort": "stable sort", "partition": "hash_partition"}
    if args.ops:
        ops = {k: v for k, v in ops.items() if any(k.startswith(wanted[o]) for o in args.ops.split(","))}
    for name, (fn, algo) in ops.items():
        ms, rows, kern = _profiled(N, fn, args.steps)
        print(json.dumps({"workload": f"{name}: {n} rows", "ms": round(ms, 3), "rows_per_s": n / (ms / 1e3),
                          "out_rows": rows, "op_GBps_algorithmic": algo / (ms / 1e3) / 1e9,
                          "op_frac_of_peak": algo / (ms / 1e3) / 1e9 / peak, "peak_kind": kind,
                          "kernels_ms": kern}), flush=True)
    return 0


def run_sort_workload(args):
    """--rows (default 100M) rows: uniform random int64 key over
    [-2^62, 2^62) and an int32 payload; stable ascending sort on the key."""
    import pyarrow as pa
    import torch

    from legate_dataframe import LogicalColumn, LogicalTable
    from legate_dataframe import _native as N
    from legate_dataframe.lib.sort import sort

    dev = torch.device("cuda", 0)
    n = args.rows
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    k = torch.randint(-(2**62), 2**62, (n,), device=dev, generator=g)
    v = torch.arange(n, device=dev, dtype=torch.int32)
    t = LogicalTable([LogicalColumn.from_torch(k, pa.int64()), LogicalColumn.from_torch(v, pa.int32())], ["k", "v"])
    algo = 2 * n * 12  # key + payload in, sorted table out
    peak, kind = measured_peak_gbs()
    ms, rows, kern = _profiled(N, lambda: sort(t, ["k"], stable=True), args.steps)
    print(json.dumps({"workload": f"stable sort (int64 key, int32 payload): {n} rows", "ms": round(ms, 3),
                      "rows_per_s": n / (ms / 1e3), "out_rows": rows,
                      "op_GBps_algorithmic": algo / (ms / 1e3) / 1e9,
                      "op_frac_of_peak": algo / (ms / 1e3) / 1e9 / peak, "peak_kind": kind,
                      "kernels_ms": kern}), flush=True)
    return 0


def run_ingest_workload(args):
    """--rows (default 20M) rows as a host Arrow table shaped like the string
    workload (string key from a 2M-entry dictionary, 10% null int64 ts,
    float32 value) into the device layout: `LogicalTable.from_arrow` (Arrow
    buffers copied as they are, bitmaps and offsets expanded on the device)
    against the same conversion done on the host with numpy and then copied;
    and `parquet_read` of the table written to a local Parquet file against
    Arrow's Parquet read alone."""
    import numpy as np
    import pyarrow as pa
    import pyarrow.parquet as pq
    import torch

    from legate_dataframe import LogicalColumn, LogicalTable
    from legate_dataframe.lib.parquet import parquet_read

    dev = torch.device("cuda", 0)
    n, nd = args.rows, 2_000_000
    rng = np.random.default_rng(9)
    lens = rng.integers(8, 25, nd)
    alphabet = np.frombuffer(b"abcdefghijklmnopqrstuvwxyz0123456789", dtype=np.uint8)
    chars = alphabet[rng.integers(0, 36, int(lens.sum()))]
    doff = np.zeros(nd + 1, np.int32)
    np.cumsum(lens, out=doff[1:])
    dictionary = pa.StringArray.from_buffers(nd, pa.py_buffer(doff), pa.py_buffer(chars.tobytes()))
    ranks = np.minimum(rng.zipf(1.5, n), nd) - 1
    key = pa.DictionaryArray.from_arrays(pa.array(ranks.astype(np.int32)), dictionary).cast(pa.string())
    ts = pa.array(rng.integers(0, 365 * 86400 * 10**6, n), mask=rng.random(n) < 0.10)
    val = pa.array(rng.lognormal(size=n).astype(np.float32))
    t = pa.table({"k": key, "ts": ts, "v": val})
    arrow_bytes = sum(b.size for c in t.columns for ch in c.chunks for b in ch.buffers() if b is not None)

    def host_then_copy():
        cols = []
        for c in t.columns:
            h = LogicalColumn.from_arrow(c, device=torch.device("cpu"))
            cols.append(LogicalColumn(h.arrow_type, h.ldf_type, h.size, h.data.to(dev),
                                      None if h.valid is None else h.valid.to(dev),
                                      None if h.chars is None else h.chars.to(dev), h.chars_base, h.num_chars))
        return LogicalTable(cols, t.column_names)

    def timed(fn, steps):
        fn()
        torch.cuda.synchronize()
        best = []
        for _ in range(steps):
            t0 = time.perf_counter()
            r = fn()
            torch.cuda.synchronize()
            best.append(time.perf_counter() - t0)
            del r
        return 1e3 * statistics.median(best)

    steps = max(args.steps, 3)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "t.parquet")
        pq.write_table(t, path)
        results = {
            "from_arrow (device expansion)": timed(lambda: LogicalTable.from_arrow(t), steps),
            "host numpy conversion + copy": timed(host_then_copy, steps),
            "parquet_read": timed(lambda: parquet_read(path), steps),
            "Arrow Parquet read alone (host)": timed(lambda: pq.read_table(path), steps),
        }
    for name, ms in results.items():
        print(json.dumps({"workload": f"ingest {name}: {n} rows", "ms": round(ms, 3), "rows_per_s": n / (ms / 1e3),
                          "arrow_GBps": arrow_bytes / (ms / 1e3) / 1e9, "arrow_bytes": arrow_bytes,
                          "timing": "host wall clock, median, device synchronized"}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rows", type=int, default=N_ROWS)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-sample", type=int, default=4_000_000)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--served-requests", type=int, default=8192)
    ap.add_argument("--ref-rows", type=int, default=8_000_000, help="rows per step of the reference arm")
    ap.add_argument("--ops", default="", help="--workload strings: comma list of groupby,sort,partition (default all)")
    ap.add_argument("--workload", default="groupby", choices=["groupby", "join", "strings", "sort", "ingest"],
                    help="groupby = the benchmark line; join / strings / sort / ingest print per-op lines")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "groupby":
        if args.rows == N_ROWS and args.workload in ("strings", "sort", "ingest"):
            args.rows = 20_000_000 if args.workload == "ingest" else 100_000_000
        if args.workload == "ingest":
            return run_ingest_workload(args)
        if args.workload == "sort":
            return run_sort_workload(args)
        return run_join_workload(args) if args.workload == "join" else run_strings_workload(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=device)

    from legate_dataframe import _native as N
    from legate_dataframe.lib.groupby_aggregation import groupby_aggregation

    N.lib()
    n = args.rows
    keys, v, valid, i = make_input_device(n, device)
    table = device_table(keys, v, valid, i)

    def step():
        return groupby_aggregation(table, ["k"], AGGS)

    for _ in range(max(args.warmup, 3)):
        out = step()
    groups = out.num_rows()
    out_b = output_bytes(out)
    del out
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- timed region (device-resident inputs) -----------------------------
    launches0 = N.launch_count()
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record()
        for _ in range(args.steps):
            out = step()
            del out
        ev1.record()
        torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1), world, device)
    launches = (N.launch_count() - launches0) // args.steps
    ms_step = ms / args.steps
    value = world * n / (ms_step / 1e3)

    # ---- per-kernel device times (CUDA events on the launching stream) ------
    N.profile_enable(True)
    N.profile_report(reset=True)
    for _ in range(2):
        out = step()
        del out
    torch.cuda.synchronize()
    prof = N.profile_report(reset=True)
    N.profile_enable(False)
    # algorithmic bytes each kernel streams per launch (the input columns it
    # reads once): assign reads the keys, the column kernels the float64 value
    # + its null mask or the int32 value, nunique the int32 value
    per_launch_bytes = {
        "assign": 8 * n,
        "column": (9 * n + 4 * n) / 2,
        "nunique": 4 * n,
    }
    total_prof = sum(t for _, t in prof.values())
    dom = max((k for k in prof if k in per_launch_bytes), key=lambda k: prof[k][1], default=None)
    peak, peak_kind = measured_peak_gbs()
    if dom is not None:
        dom_cnt, dom_ms = prof[dom]
        dom_ms /= max(dom_cnt, 1)
        algo_kernel = per_launch_bytes[dom]
        achieved = algo_kernel / (dom_ms / 1e3) / 1e9
    else:
        dom_ms, algo_kernel, achieved = float("nan"), 0, float("nan")
    traffic = None
    tp = ROOT / "profiles" / f"groupby_config1_{dom}_traffic.json"
    if tp.exists():
        try:
            tj = json.loads(tp.read_text())
            traffic = float(tj["dram_bytes_per_row"]) * n
        except (KeyError, ValueError):
            traffic = None
    op_bytes = n * IN_BYTES_PER_ROW + out_b

    # ---- end to end: host (pinned) -> device -> op -> host -----------------
    e2e = None
    if rank == 0 or world > 1:
        hk = torch.empty(n, dtype=torch.int64, pin_memory=True)
        hv = torch.empty(n, dtype=torch.float64, pin_memory=True)
        hm = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        hi = torch.empty(n, dtype=torch.int32, pin_memory=True)
        hk.copy_(keys)
        hv.copy_(v)
        hm.copy_(valid)
        hi.copy_(i)
        torch.cuda.synchronize()
        d2h = 0

        def e2e_step():
            # the table's columns are pinned host memory: the op copies each
            # to the device itself, overlapping the copies with its passes
            res = groupby_aggregation(device_table(hk, hv, hm, hi), ["k"], AGGS)
            res.to_arrow()
            return output_bytes(res)

        e2e_step()  # warm-up: the pinned staging buffer of to_arrow is allocated once
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record()
        for _ in range(args.e2e_steps):
            d2h = e2e_step()
        e1.record()
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.e2e_steps, world, device)
        e2e = {"value": world * n / (e2e_ms / 1e3), "unit": "rows/s", "ms_per_step": e2e_ms,
               "h2d_bytes_per_step": n * IN_BYTES_PER_ROW, "d2h_bytes_per_step": d2h}
        del hk, hv, hm, hi

    # ---- CPU baseline (rank 0, N=1 only) ------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        import pyarrow as pa

        sample = host_sample(keys, v, valid, i, min(args.cpu_sample, n))
        rate, el, reps = cpu_groupby_rate(sample, use_threads=False)
        cpu = {"value": rate, "unit": "rows/s", "cores": 1, "kind": "port",
               "sample": f"first {sample.num_rows} rows of the same input x{reps} ({el:.1f} s); Arrow "
                         f"{pa.__version__} Acero aggregate hash_sum/mean/count_all/count/min/max/count_distinct, "
                         "use_threads=False: the Arrow calls of the reference's cpu_variant (one legate CPU task)"}

    # ---- served mix (rank 0, N=1 only) --------------------------------------
    served = None
    if rank == 0 and world == 1 and not args.no_served:
        del keys, v, valid, i, table
        torch.cuda.empty_cache()
        served = run_served(device, args.served_requests)

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "rows/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": max(args.warmup, 3),
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64+int64 (fixed-point exact f64 sums)",
        "data": "synthetic (seeded on device: Zipf(1.1) keys over 10M int64, f64 N(0,1) 10% nulls, i32 U[0,1e6))",
        "config": {"workload": "groupby config 1: 200M rows; SUM/MEAN(f64), COUNT(*), COUNT(f64), MIN/MAX(i32), "
                               "NUNIQUE(i32)", "rows": n, "groups": groups,
                   "l2": "inputs 4.2 GB >> 126 MB L2 (no flush needed)", "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "algorithmic_bytes": algo_kernel, "kernel_ms": dom_ms,
                     "op_frac": (op_bytes / (ms_step / 1e3) / 1e9) / peak, "op_algorithmic_bytes": op_bytes},
        "kernel_ms": {k: round(t / max(c, 1), 4) for k, (c, t) in prof.items()},
        "kernel_share": {k: round(t / total_prof, 4) for k, (c, t) in prof.items()} if total_prof else {},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "e2e": e2e,
        "cpu_baseline": cpu,
        "served": served,
    }
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
