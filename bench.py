"""Benchmark of the B200 relational hot path.

The headline line is hash groupby aggregation, 200M rows (Zipf(1.1) int64
keys over 10M distinct values; float64 N(0,1) with 10% nulls; int32
U[0, 1e6)); SUM and MEAN of the float64 column, COUNT(*) and COUNT of the
float64 column, MIN/MAX and NUNIQUE of the int32 column.  One step = one
groupby_aggregation call through the public API (C ABI) on device-resident
inputs (4.2 GB, far larger than the 126 MB L2, so no flush is needed).  The
step's result is checked outside the timed region (`parity`).

At N=1 the same JSON line also carries
  * `joins`: inner / left / full hash joins, 200M probe x 20M build rows
    (int32 keys, 5% null probe keys, Zipf(0.9) hits);
  * `strings`: 100M string-key rows: groupby SUM/COUNT(*), stable sort
    (key asc, ts desc), hash_partition into 256 buckets;
  * `csv` / `parquet`: csv_read / parquet_read of a 4M-row file of the
    string workload's shape on the device readers, against Arrow's readers on
    the host;
  * `served`: the batched/served mix (8,192 small joins and groupbys arriving
    at 2,000 req/s) through the continuous-batching server and, for
    comparison, the same requests issued one op per launch.
(--no-joins / --no-strings / --no-csv (both files) / --no-served skip them.)

`--workload join|strings|sort|ingest` instead prints one line per op.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`--impl reference` times the reference's CPU implementation of the path (the
Arrow Acero calls of GroupByAggregationTask::cpu_variant) on the same
200M-row workload every step: the rows hash-sharded over the host cores, one
single-threaded task body per shard, all shards at once (legate --cpus N;
the shuffle itself is not timed).

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
from legate_dataframe.workloads import GROUPBY_AGGS as AGGS  # noqa: E402
IN_BYTES_PER_ROW = 8 + 8 + 1 + 4  # key + f64 + its null mask + i32 (legate layout)


def measured_peak_gbs():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return 6650.0, "fallback"


def host_table(keys, v, valid, i):
    import pyarrow as pa

    return pa.table({"k": keys.cpu().numpy(), "v": pa.array(v.cpu().numpy(), mask=valid.cpu().numpy() == 0),
                     "i": i.cpu().numpy()})


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
# CPU side: the reference's CPU path (Arrow Acero aggregate, the calls of
# GroupByAggregationTask::cpu_variant, one single-threaded task body per
# legate CPU) on hash shards of the same workload
# ---------------------------------------------------------------------------
def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def shard_of(keys, nshards: int):
    """Hash shard of every int64 key (multiplicative hash, top bits), as
    legate's hash repartitioning sends each key's rows to one CPU task."""
    import numpy as np

    with np.errstate(over="ignore"):
        h = keys.view(np.uint64) * np.uint64(0x9E3779B97F4A7C15)
    return ((h >> np.uint64(32)) % np.uint64(nshards)).astype(np.uint8)


def reference_shards(n: int, nshards: int, threads: int):
    """The 200M-row groupby workload on the host (numpy, seeded; the same
    distributions as the device generator), cut into `nshards` hash shards
    of the key: a list of Arrow tables.  Rows are generated in chunks on
    `threads` threads; each chunk is split by shard, and a shard's table is
    the concatenation of its pieces (no further copy)."""
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np
    import pyarrow as pa

    from legate_dataframe import workloads as W

    nk = W.GROUPBY_KEYS
    cdf = np.cumsum(np.arange(1, nk + 1, dtype=np.float64) ** -1.1)
    cdf /= cdf[-1]
    key_values = np.random.default_rng(3).permutation(nk).astype(np.int64) * 2_654_435_761 + 12_345
    nchunks = max(threads, 1)
    bounds = [n * c // nchunks for c in range(nchunks + 1)]

    def chunk(c):
        m = bounds[c + 1] - bounds[c]
        rng = np.random.default_rng([1, c])
        k = key_values[np.minimum(np.searchsorted(cdf, rng.random(m)), nk - 1)]
        v = rng.normal(size=m)
        null = rng.random(m) < 0.10
        i = rng.integers(0, 1_000_000, m).astype(np.int32)
        s = shard_of(k, nshards)
        order = np.argsort(s, kind="stable")
        off = np.zeros(nshards + 1, np.int64)
        np.cumsum(np.bincount(s, minlength=nshards), out=off[1:])
        k, v, null, i = k[order], v[order], null[order], i[order]
        return [pa.table({"k": k[off[j]:off[j + 1]], "v": pa.array(v[off[j]:off[j + 1]], mask=null[off[j]:off[j + 1]]),
                          "i": i[off[j]:off[j + 1]]}) for j in range(nshards)]

    with ThreadPoolExecutor(nchunks) as ex:
        pieces = list(ex.map(chunk, range(nchunks)))
    return [pa.concat_tables([p[j] for p in pieces]) for j in range(nshards)]


def run_shards(shards, threads: int):
    """One Acero aggregate (use_threads=False: one task body) per shard, all
    shards at once on `threads` host threads (Acero releases the GIL)."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import arrow_ref

    with ThreadPoolExecutor(threads) as ex:
        return list(ex.map(lambda s: arrow_ref.groupby(s, ["k"], AGGS, use_threads=False), shards))


def run_reference(args):
    """--impl reference: the reference's CPU implementation of the path on the
    full 200M-row workload every step, with every host core."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import pyarrow as pa

    world = int(os.environ.get("WORLD_SIZE", "1"))
    n = args.rows
    cores = host_cores()
    shards = reference_shards(n, cores, cores)
    for _ in range(args.warmup):
        run_shards(shards, cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        res = run_shards(shards, cores)
    el = time.perf_counter() - t0
    groups = sum(r.num_rows for r in res)
    rate = n * args.steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "rows/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+int64",
        "data": "synthetic (seeded on the host with numpy: the workload's distributions)",
        "config": groupby_config(n, world),
        "groups": groups,
        "cpu_baseline": {"value": rate, "unit": "rows/s", "cores": cores, "kind": "port",
                         "sample": f"every step the whole {n}-row workload: {cores} hash shards of the key, one "
                                   f"Arrow {pa.__version__} Acero aggregate (hash_sum/mean/count_all/count/min/max/"
                                   "count_distinct, use_threads=False: one cpu_variant task body) per shard, "
                                   f"{cores} shards at once on {cores} host threads (legate --cpus {cores}); "
                                   "the shuffle into shards is not timed"},
        "e2e": {"value": rate, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def groupby_config(n: int, world: int) -> dict:
    return {"workload": "hash groupby, 200M rows; int64 Zipf(1.1) keys over 10M values, f64 N(0,1) 10% nulls, "
                        "i32 U[0,1e6); SUM/MEAN(f64), COUNT(*), COUNT(f64), MIN/MAX(i32), NUNIQUE(i32)",
            "rows": n, "l2": "inputs 4.2 GB >> 126 MB L2 (no flush needed)", "parallelism": f"replicas x{world}"}


def cpu_task_rate(keys, v, valid, i, nshards: int, min_seconds: float = 10.0):
    """One legate CPU task's rate: shard 0 of `nshards` hash shards of the
    device input (the same rows the GPU step aggregates) through one Acero
    aggregate with use_threads=False, repeated for >= min_seconds."""
    import numpy as np

    from oracle import arrow_ref

    host = host_table(keys, v, valid, i)
    sel = np.nonzero(shard_of(host.column("k").to_numpy(), nshards) == 0)[0]
    sample = host.take(sel)
    del host
    t0 = time.perf_counter()
    reps = 0
    while True:
        arrow_ref.groupby(sample, ["k"], AGGS, use_threads=False)
        reps += 1
        el = time.perf_counter() - t0
        if el >= min_seconds or reps >= 20:
            break
    return sample.num_rows * reps / el, sample.num_rows, el, reps


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
# the joins and the string workload (sub-records of the default line, or one
# line per op with --workload join / strings): device ms of the op (CUDA
# events on the stream), rows/s, the op's algorithmic bytes against the
# measured HBM peak, and per-kernel device ms
# ---------------------------------------------------------------------------
def _profiled(N, fn, steps):
    import torch

    for _ in range(2):
        r = fn()
        del r
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        r = fn()
        del r
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    N.profile_enable(True)
    N.profile_report(reset=True)
    r = fn()
    torch.cuda.synchronize()
    prof = N.profile_report(reset=True)
    N.profile_enable(False)
    return ms, r, {k: [c, round(t, 4)] for k, (c, t) in sorted(prof.items(), key=lambda kv: -kv[1][1])}


def _record(name, ms, rows_in, out_rows, algo, kern, peak, kind):
    total = sum(t for _, t in kern.values()) or 1.0
    dom = next(iter(kern), None)
    return {"op": name, "ms": round(ms, 4), "rows_per_s": rows_in / (ms / 1e3), "out_rows": out_rows,
            "algorithmic_bytes": int(algo), "GBps": algo / (ms / 1e3) / 1e9,
            "frac": algo / (ms / 1e3) / 1e9 / peak, "peak_kind": kind,
            "dominant_kernel": dom, "dominant_ms": kern[dom][1] if dom else None,
            "dominant_share": round(kern[dom][1] / total, 4) if dom else None, "kernels_ms": kern}


_C1 = 0xFF51AFD7ED558CCD - (1 << 64)
_C2 = 0xC4CEB9FE1A85EC53 - (1 << 64)


def _mix(x):
    m31 = (1 << 31) - 1
    x = x ^ ((x >> 33) & m31)
    x = x * _C1
    x = x ^ ((x >> 33) & m31)
    x = x * _C2
    return x ^ ((x >> 33) & m31)


def _row_checksum(cols):
    """Order-independent checksum of rows given as (int64 bits, valid) columns."""
    import torch

    h = None
    for j, (x, ok) in enumerate(cols):
        a = torch.where(ok, _mix(x + (j + 1) * 0x9E3779B9), torch.full_like(x, 0x5BD1E995 + j))
        h = a if h is None else _mix(h + a)
    m = 0xFFFFFFFF
    return int((h & m).sum()), int(((h >> 32) & m).sum()), [int(ok.sum()) for _, ok in cols]


def _col_bits(c):
    import torch

    from legate_dataframe import _native as N

    n = c.size
    w = N.TYPE_WIDTH[c.ldf_type]
    x = c.data[: n * w].view({1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}[w]).to(torch.int64)
    ok = c.valid[:n].bool() if c.valid is not None else torch.ones(n, dtype=torch.bool, device=x.device)
    return x, ok


def _join_expected(J, how):
    """The join's rows by definition (unique build keys: a probe row with a
    valid key matches the build row holding that key), as (bits, valid)."""
    import torch

    dev = J.bkey.device
    nb = J.bkey.numel()
    inv = torch.empty(nb, dtype=torch.int64, device=dev)
    inv[J.bkey.long()] = torch.arange(nb, device=dev)
    inr = J.pvalid & (J.pkey >= 0) & (J.pkey < nb)
    brow = torch.where(inr, inv[J.pkey.long().clamp(0, nb - 1)], torch.full_like(inv[:1], -1))
    hit = brow >= 0
    one = torch.ones_like(hit)
    safe = brow.clamp(min=0)
    cols = [(J.pkey.to(torch.int64), J.pvalid), (J.ppay.view(torch.int64), one),
            (J.bkey[safe].to(torch.int64), hit), (J.bp1[safe], hit), (J.bp2[safe], hit)]
    if how == "inner":
        return [(x[hit], one[hit]) for x, _ in cols]
    if how == "left":
        return cols
    used = torch.zeros(nb, dtype=torch.bool, device=dev)
    used[brow[hit]] = True
    un = torch.nonzero(~used).squeeze(1)
    z = torch.zeros(un.numel(), dtype=torch.int64, device=dev)
    f = torch.zeros(un.numel(), dtype=torch.bool, device=dev)
    t = ~f
    tail = [(z, f), (z, f), (J.bkey[un].to(torch.int64), t), (J.bp1[un], t), (J.bp2[un], t)]
    return [(torch.cat([a, b]), torch.cat([m, mb])) for (a, m), (b, mb) in zip(cols, tail)]


def join_records(steps: int, n_probe: int, n_build: int = 20_000_000, check: bool = True):
    """Inner / left / full join of the 200M x 20M int32-key workload."""
    import torch

    from legate_dataframe import _native as N
    from legate_dataframe import workloads as W
    from legate_dataframe.lib.join import JoinType, join

    dev = torch.device("cuda", torch.cuda.current_device())
    J = W.int32_join(n_probe, n_build, dev)
    lt, rt = J.tables()
    peak, kind = measured_peak_gbs()
    out = []
    for jt in (JoinType.INNER, JoinType.LEFT, JoinType.FULL):
        ms, res, kern = _profiled(N, lambda: join(lt, rt, lhs_keys=["lk"], rhs_keys=["rk"], join_type=jt), steps)
        algo = n_build * 20 + n_probe * 13 + output_bytes(res)
        rec = _record(f"join {jt.name.lower()}: {n_probe} probe x {n_build} build rows (int32 keys)", ms,
                      n_probe + n_build, res.num_rows(), algo, kern, peak, kind)
        if check:
            got = _row_checksum([_col_bits(c) for c in res.get_columns()])
            rec["parity"] = "ok" if got == _row_checksum(_join_expected(J, jt.name.lower())) else "MISMATCH"
        del res
        out.append(rec)
    del J, lt, rt
    torch.cuda.empty_cache()
    return out


def string_records(steps: int, n: int, ops: str = ""):
    """groupby SUM/COUNT(*) on the string key, stable sort (key asc, ts
    desc), hash_partition(key, 256) of the 100M-row string workload."""
    import torch

    from legate_dataframe import _native as N
    from legate_dataframe import workloads as W
    from legate_dataframe.lib.groupby_aggregation import groupby_aggregation
    from legate_dataframe.lib.hash_partition import hash_partition
    from legate_dataframe.lib.sort import sort

    dev = torch.device("cuda", torch.cuda.current_device())
    S = W.string_rows(n, dev)
    t = S.table()
    nchars = S.chars.numel()
    row_bytes = 16 + nchars / n + 8 + 4
    todo = {
        "groupby SUM/COUNT(*) on the string key": (
            lambda: groupby_aggregation(t, ["k"], [("v", "sum", "s"), (None, "count_all", "c")]),
            n * (16 + nchars / n + 4)),
        "stable sort (key asc, ts desc)": (
            lambda: sort(t, ["k", "ts"], sort_ascending=[True, False], stable=True), 2 * n * row_bytes),
        "hash_partition(key, 256)": (lambda: hash_partition(t, ["k"], 256), 2 * n * row_bytes),
    }
    wanted = {"groupby": "groupby", "sort": "stable sort", "partition": "hash_partition"}
    if ops:
        todo = {k: v for k, v in todo.items() if any(k.startswith(wanted[o]) for o in ops.split(","))}
    peak, kind = measured_peak_gbs()
    out = []
    for name, (fn, algo) in todo.items():
        ms, res, kern = _profiled(N, fn, steps)
        tbl = res[0] if isinstance(res, tuple) else res
        if name.startswith("groupby"):
            algo += output_bytes(tbl) + sum(int(c.num_chars) for c in tbl.get_columns() if c.chars is not None)
        out.append(_record(f"{name}: {n} rows", ms, n, tbl.num_rows(), algo, kern, peak, kind))
        del res, tbl
    del S, t
    torch.cuda.empty_cache()
    return out


def run_join_workload(args):
    for rec in join_records(args.steps, args.rows, check=False):
        print(json.dumps(rec), flush=True)
    return 0


def run_strings_workload(args):
    for rec in string_records(args.steps, args.rows, args.ops):
        print(json.dumps(rec), flush=True)
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
    ms, res, kern = _profiled(N, lambda: sort(t, ["k"], stable=True), args.steps)
    print(json.dumps(_record(f"stable sort (int64 key, int32 payload): {n} rows", ms, n, res.num_rows(), algo, kern,
                             peak, kind)), flush=True)
    return 0


def _string_workload_table(n: int, seed: int = 9):
    """n rows shaped like the 100M-row string workload, on the host: string
    key from a 2M-entry dictionary (Zipf), 10% null int64 ts, float32 value."""
    import numpy as np
    import pyarrow as pa

    nd = 2_000_000
    rng = np.random.default_rng(seed)
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
    return pa.table({"k": key, "ts": ts, "v": val})


def csv_record(n: int, steps: int = 3) -> dict:
    """csv_read of an n-row CSV file of the string workload's shape (local
    file, page cache warm): the device reader end to end (file -> pinned
    memory -> device -> parsed columns), its kernels, and the reference's
    CPU reader on the same file (Arrow read_csv, use_threads=False as in
    CSVRead::cpu_variant, and with all host threads); parity against Arrow."""
    import pyarrow as pa
    import pyarrow.csv as pacsv
    import torch

    from legate_dataframe import _native as N
    from legate_dataframe.lib.csv import csv_read

    t = _string_workload_table(n)
    names, dtypes = t.column_names, [pa.string(), pa.int64(), pa.float32()]
    conv = pacsv.ConvertOptions(column_types=dict(zip(names, dtypes)), strings_can_be_null=True,
                                quoted_strings_can_be_null=True)

    def wall(fn):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            t0 = time.perf_counter()
            r = fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
            del r
        return statistics.median(ts)

    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "t.csv")
        pacsv.write_csv(t, path)
        size = os.path.getsize(path)
        dev_s = wall(lambda: csv_read(path, dtypes=dtypes, names=names))
        N.profile_enable(True)
        N.profile_report(reset=True)
        got = csv_read(path, dtypes=dtypes, names=names)
        torch.cuda.synchronize()
        prof = N.profile_report(reset=True)
        N.profile_enable(False)
        one = wall(lambda: pacsv.read_csv(path, read_options=pacsv.ReadOptions(use_threads=False),
                                          convert_options=conv))
        allt = wall(lambda: pacsv.read_csv(path, convert_options=conv))
        exp = pacsv.read_csv(path, parse_options=pacsv.ParseOptions(newlines_in_values=True), convert_options=conv)
        parity = "ok" if got.to_arrow().equals(exp.select(names)) else "MISMATCH"
    kernel_ms = sum(v[1] for v in prof.values())
    return {"op": f"csv_read: {n} rows, {size} bytes (string key, nullable int64, float32)",
            "ms": round(dev_s * 1e3, 3), "GBps_text": size / dev_s / 1e9, "rows_per_s": n / dev_s,
            "kernel_ms": round(kernel_ms, 3), "kernel_GBps_text": size / (kernel_ms / 1e3) / 1e9,
            "kernels_ms": {k: [c, round(ms, 4)] for k, (c, ms) in sorted(prof.items(), key=lambda kv: -kv[1][1])},
            "arrow_1_thread_ms": round(one * 1e3, 3), "arrow_all_threads_ms": round(allt * 1e3, 3),
            "host_threads": host_cores(), "vs_arrow_1_thread": one / dev_s, "vs_arrow_all_threads": allt / dev_s,
            "parity": parity, "timing": "host wall clock, median, device synchronized; file in the page cache"}


def parquet_record(n: int, steps: int = 3) -> dict:
    """parquet_read of an n-row Parquet file of the string workload's shape
    (Arrow's writer defaults: Snappy, dictionary pages, page cache warm): the
    device decoder end to end (file -> pinned memory -> device -> decoded
    columns), its kernels, and the reference's CPU reader on the same file
    (Arrow read_table with one thread, and with all host threads); parity
    against Arrow."""
    import pyarrow.parquet as pq
    import torch

    from legate_dataframe import _native as N
    from legate_dataframe.lib.parquet import parquet_read

    t = _string_workload_table(n)

    def wall(fn):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            t0 = time.perf_counter()
            r = fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
            del r
        return statistics.median(ts)

    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "t.parquet")
        pq.write_table(t, path)
        size = os.path.getsize(path)
        dev_s = wall(lambda: parquet_read(path))
        N.profile_enable(True)
        N.profile_report(reset=True)
        got = parquet_read(path)
        torch.cuda.synchronize()
        prof = N.profile_report(reset=True)
        N.profile_enable(False)
        one = wall(lambda: pq.read_table(path, use_threads=False))
        allt = wall(lambda: pq.read_table(path))
        parity = "ok" if got.to_arrow().equals(pq.read_table(path)) else "MISMATCH"
    kernel_ms = sum(v[1] for v in prof.values())
    out_bytes = sum(c.size * N.TYPE_WIDTH[c.ldf_type] + (c.size if c.valid is not None else 0) + (c.num_chars or 0)
                    for c in got.get_columns())
    return {"op": f"parquet_read: {n} rows, {size} bytes of Parquet (Snappy, dictionary pages; string key, "
                  "nullable int64, float32)",
            "ms": round(dev_s * 1e3, 3), "rows_per_s": n / dev_s, "file_GBps": size / dev_s / 1e9,
            "kernel_ms": round(kernel_ms, 3), "output_bytes": out_bytes,
            "kernels_ms": {k: [c, round(ms, 4)] for k, (c, ms) in sorted(prof.items(), key=lambda kv: -kv[1][1])},
            "arrow_1_thread_ms": round(one * 1e3, 3), "arrow_all_threads_ms": round(allt * 1e3, 3),
            "host_threads": host_cores(), "vs_arrow_1_thread": one / dev_s, "vs_arrow_all_threads": allt / dev_s,
            "parity": parity, "timing": "host wall clock, median, device synchronized; file in the page cache"}


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
    n = args.rows
    t = _string_workload_table(n)
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
    print(json.dumps(csv_record(n, steps)), flush=True)
    print(json.dumps(parquet_record(n, steps)), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rows", type=int, default=N_ROWS)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--served-requests", type=int, default=8192)
    ap.add_argument("--no-joins", action="store_true")
    ap.add_argument("--no-strings", action="store_true")
    ap.add_argument("--no-csv", action="store_true")
    ap.add_argument("--sub-steps", type=int, default=5, help="timed steps of each join / string op record")
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
    from legate_dataframe import workloads as W
    from legate_dataframe.lib.groupby_aggregation import groupby_aggregation

    N.lib()
    n = args.rows
    keys, v, valid, i = W.zipf_groupby(n, device)
    table = W.groupby_table(keys, v, valid, i)

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
    torch.cuda.synchronize()
    prof = N.profile_report(reset=True)
    N.profile_enable(False)

    # ---- the step's result, checked outside the timed region ----------------
    parity = {"groupby": groupby_parity(keys, v, valid, i, out)}
    del out
    torch.cuda.empty_cache()

    # algorithmic bytes each kernel streams per launch (the input columns it
    # reads once)
    per_launch_bytes = kernel_algorithmic_bytes(n)
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
    tp = ROOT / "profiles" / f"groupby_200m_{dom}_traffic.json"
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
            res = groupby_aggregation(W.groupby_table(hk, hv, hm, hi), ["k"], AGGS)
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

    # ---- CPU baseline (rank 0, N=1 only): one legate CPU task's shard -------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        import pyarrow as pa

        shards = host_cores()
        rate, rows, el, reps = cpu_task_rate(keys, v, valid, i, shards)
        cpu = {"value": rate, "unit": "rows/s", "cores": 1, "kind": "port",
               "sample": f"hash shard 0 of {shards} of the same {n}-row input ({rows} rows, the share of one "
                         f"legate CPU task at --cpus {shards}) x{reps} ({el:.1f} s); Arrow {pa.__version__} Acero "
                         "aggregate hash_sum/mean/count_all/count/min/max/count_distinct, use_threads=False: "
                         "the Arrow calls of the reference's cpu_variant"}
    del keys, v, valid, i, table
    torch.cuda.empty_cache()

    # ---- joins and the string workload (rank 0, N=1 only) -------------------
    joins = strings = None
    if rank == 0 and world == 1 and not args.no_joins:
        joins = join_records(args.sub_steps, 200_000_000)
    if rank == 0 and world == 1 and not args.no_strings:
        strings = string_records(args.sub_steps, 100_000_000)
    if joins is not None:
        parity["joins"] = "ok" if all(r.get("parity") == "ok" for r in joins) else "MISMATCH"

    csv = parquet = None
    if rank == 0 and world == 1 and not args.no_csv:
        csv = csv_record(4_000_000)
        parity["csv"] = csv["parity"]
        parquet = parquet_record(4_000_000)
        parity["parquet"] = parquet["parity"]

    # ---- served mix (rank 0, N=1 only) --------------------------------------
    served = None
    if rank == 0 and world == 1 and not args.no_served:
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
        "config": groupby_config(n, world),
        "groups": groups,
        "parity": parity,
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
        "joins": joins,
        "strings": strings,
        "csv": csv,
        "parquet": parquet,
        "served": served,
    }
    print(json.dumps(line))
    return 0


def kernel_algorithmic_bytes(n: int) -> dict:
    """Algorithmic bytes per launch of the groupby's row passes: the input
    columns each reads once (assign the keys; the column passes the float64
    value + its null mask or the int32 value; nunique the int32 value)."""
    return {"assign": 8 * n, "column": (9 * n + 4 * n) / 2, "nunique": 4 * n}


def groupby_parity(keys, v, valid, i, out) -> str:
    """The step's result against the aggregates recomputed with torch's sorts
    (rows sorted by key, then by the int32 value inside a key): COUNT(*),
    COUNT, MIN, MAX and NUNIQUE exact; SUM and MEAN within the rounding bound
    of an fp64 sum in any order ((count + 2) x 2^-52 x the sum of |x|)."""
    import torch

    n = keys.numel()
    p = torch.sort(i, stable=True).indices
    perm = p[torch.sort(keys[p], stable=True).indices]
    del p
    sk, si = keys[perm], i[perm]
    sm = valid[perm].bool()
    sv = torch.where(sm, v[perm], torch.zeros((), dtype=v.dtype, device=v.device))
    del perm
    uniq, counts = torch.unique_consecutive(sk, return_counts=True)
    g = uniq.numel()
    end = torch.cumsum(counts, 0)
    start = end - counts
    seg = torch.repeat_interleave(torch.arange(g, device=keys.device), counts)
    new = torch.ones(n, dtype=torch.int64, device=keys.device)
    new[1:] = ((si[1:] != si[:-1]) | (sk[1:] != sk[:-1])).to(torch.int64)
    del sk
    zeros = torch.zeros(g, dtype=torch.int64, device=keys.device)
    nd = zeros.clone().index_add_(0, seg, new)
    cv = zeros.clone().index_add_(0, seg, sm.to(torch.int64))
    fz = torch.zeros(g, dtype=torch.float64, device=keys.device)
    s = fz.clone().index_add_(0, seg, sv)
    a = fz.clone().index_add_(0, seg, sv.abs())
    mn, mx = si[start], si[end - 1]
    del si, sm, sv, seg, new

    cols = dict(zip(out.get_column_names(), out.get_columns()))

    def col(name, dt):
        c = cols[name]
        return c.data[: c.size * torch.empty((), dtype=dt).element_size()].view(dt), \
            (c.valid[: c.size].bool() if c.valid is not None else None)

    k, _ = col("k", torch.int64)
    if k.numel() != g:
        return f"MISMATCH: {k.numel()} groups, expected {g}"
    o = torch.sort(k).indices
    bad = []
    if not torch.equal(k[o], uniq):
        bad.append("k")
    for name, dt, want in (("count", torch.int64, counts), ("count_v", torch.int64, cv), ("min_i", torch.int32, mn),
                           ("max_i", torch.int32, mx), ("nunique_i", torch.int64, nd)):
        x, _ = col(name, dt)
        if not torch.equal(x[o].to(want.dtype), want):
            bad.append(name)
    has = cv > 0
    bound = (cv.to(torch.float64) + 2) * 2.0**-52 * a + 1e-300
    for name, want, lim in (("sum_v", s, bound), ("mean_v", s / cv.clamp(min=1), bound / cv.clamp(min=1))):
        x, ok = col(name, torch.float64)
        x, ok = x[o], ok[o] if ok is not None else torch.ones_like(has)
        if not torch.equal(ok, has) or not bool(((x - want).abs() <= lim)[has].all()):
            bad.append(name)
    return "ok" if not bad else "MISMATCH: " + ",".join(bad)


if __name__ == "__main__":
    sys.exit(main())
