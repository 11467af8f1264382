"""Batched and served execution of many small joins and groupbys.

* ``BatchEngine``   ctypes wrapper of the C-ABI batch engine: a batch of
  requests runs as ONE replay of a captured CUDA graph (descriptor staging +
  three persistent kernels + status download).
* ``DeviceArena``   first-fit allocator over one device buffer; hash tables
  and outputs of admitted requests live here.
* ``Server``        request loop: tables stay resident on the device, requests
  are admitted by their projected hash-table + output bytes, and two engine
  slots on two streams run batches back to back, so requests that arrive while
  a batch is on the GPU form the next batch (continuous batching).  Reports
  throughput and p50/p99 latency (arrival -> result).
* ``Autotuner``     picks tile rows, CTAs per SM and table load factor on a
  calibration batch and persists the choice.
* ``run_one_op_per_launch``  the baseline: the same requests through the
  per-op API, one at a time.

Request kinds (config of the served benchmark): int64-key groupby with SUM +
COUNT(*) of an int64 or float64 value, and int64-key inner join with one int64
payload per side.
"""

from __future__ import annotations

import bisect
import ctypes
import json
import os
import time
from collections import deque
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional

import numpy as np
import pyarrow as pa
import torch

from legate_dataframe import _native as N

GROUPBY, JOIN = 0, 1
V_INT64, V_FLOAT64 = 0, 1


class ldf_batch_request(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32), ("vtype", ctypes.c_int32),
        ("n", ctypes.c_int64), ("m", ctypes.c_int64),
        ("k1", ctypes.c_void_p), ("v1", ctypes.c_void_p), ("k2", ctypes.c_void_p), ("v2", ctypes.c_void_p),
        ("vvalid", ctypes.c_void_p), ("table", ctypes.c_void_p), ("cap", ctypes.c_uint64),
        ("o0", ctypes.c_void_p), ("o1", ctypes.c_void_p), ("o2", ctypes.c_void_p), ("o3", ctypes.c_void_p),
        ("out_cap", ctypes.c_int64),
    ]


def _bind(L):
    if getattr(L, "_ldf_batch_bound", False):
        return L
    L.ldf_b200_batch_create.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32,
                                        ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    L.ldf_b200_batch_run.argtypes = [ctypes.c_void_p, ctypes.POINTER(ldf_batch_request), ctypes.c_int32]
    L.ldf_b200_batch_wait.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int32)]
    L.ldf_b200_batch_destroy.argtypes = [ctypes.c_void_p]
    for f in ("ldf_b200_batch_create", "ldf_b200_batch_run", "ldf_b200_batch_wait", "ldf_b200_batch_destroy"):
        getattr(L, f).restype = ctypes.c_int
    L._ldf_batch_bound = True
    return L


# ---------------------------------------------------------------------------
# requests
# ---------------------------------------------------------------------------
@dataclass
class Request:
    """One query on device-resident tables.

    groupby: ``k1`` int64 keys, ``v1`` int64/float64 values, ``valid`` optional
             bool mask of ``v1`` -> (key, sum, count) with count = valid values
    join:    ``k1``/``v1`` lhs key/payload (probe), ``k2``/``v2`` rhs (build)
             -> (lhs key, lhs payload, rhs key, rhs payload)
    ``ndv_hint`` is the expected number of distinct keys (sizes the table and
    the projected output; a wrong hint only costs a fallback re-run).
    """

    kind: int
    k1: torch.Tensor
    v1: torch.Tensor
    k2: Optional[torch.Tensor] = None
    v2: Optional[torch.Tensor] = None
    valid: Optional[torch.Tensor] = None
    ndv_hint: int = 0
    arrival: float = 0.0
    rid: int = 0
    t_in: float = 0.0  # arrival time used by the current run (0 when saturated)
    # filled when admitted / completed
    table_off: int = -1
    out_off: int = -1
    cap: int = 0
    out_cap: int = 0
    table_bytes: int = 0
    out_bytes: int = 0
    result: Optional[pa.Table] = None
    rows_out: int = 0
    done: float = 0.0
    fallback: bool = False

    @property
    def vtype(self) -> int:
        return V_FLOAT64 if self.v1.dtype == torch.float64 else V_INT64

    @property
    def n(self) -> int:
        return int(self.k1.numel())

    @property
    def m(self) -> int:
        return int(self.k2.numel()) if self.k2 is not None else 0

    @property
    def rows(self) -> int:
        return self.n + self.m

    def plan(self, load_factor: float):
        """Table capacity, output capacity and projected bytes."""
        ndv = max(1, self.ndv_hint or self.n)
        if self.kind == GROUPBY:
            groups = min(self.n, ndv)
            self.cap = max(64, int(groups / load_factor) + 1)
            stride = 8 if self.vtype == V_FLOAT64 else 3
            self.table_bytes = (self.cap + 1) * stride * 8
            self.out_cap = max(64, int(groups * 1.2) + 64)
            self.out_bytes = self.out_cap * 24
        else:
            self.cap = max(64, int(self.m / load_factor) + 1)
            self.table_bytes = self.cap * 16
            expected = self.n * self.m / ndv
            self.out_cap = max(1024, int(expected * 1.3) + 1024)
            self.out_bytes = self.out_cap * 32
        return self.table_bytes + self.out_bytes


# ---------------------------------------------------------------------------
# device arena (first fit, 256-byte aligned)
# ---------------------------------------------------------------------------
class DeviceArena:
    def __init__(self, nbytes: int, device):
        self.nbytes = int(nbytes)
        self.buf = torch.empty(self.nbytes, dtype=torch.uint8, device=device) if device is not None else None
        self._free: list[tuple[int, int]] = [(0, self.nbytes)]  # sorted (offset, size)

    @staticmethod
    def _round(n: int) -> int:
        return (int(n) + 255) & ~255

    def alloc(self, nbytes: int) -> int:
        need = self._round(max(nbytes, 1))
        for i, (off, size) in enumerate(self._free):
            if size >= need:
                if size == need:
                    self._free.pop(i)
                else:
                    self._free[i] = (off + need, size - need)
                return off
        return -1

    def release(self, off: int, nbytes: int) -> None:
        size = self._round(max(nbytes, 1))
        i = bisect.bisect_left(self._free, (off, 0))
        self._free.insert(i, (off, size))
        # coalesce with neighbours
        if i + 1 < len(self._free) and self._free[i][0] + self._free[i][1] == self._free[i + 1][0]:
            self._free[i] = (self._free[i][0], self._free[i][1] + self._free[i + 1][1])
            self._free.pop(i + 1)
        if i > 0 and self._free[i - 1][0] + self._free[i - 1][1] == self._free[i][0]:
            self._free[i - 1] = (self._free[i - 1][0], self._free[i - 1][1] + self._free[i][1])
            self._free.pop(i)

    def free_bytes(self) -> int:
        return sum(s for _, s in self._free)

    def ptr(self, off: int) -> int:
        return self.buf.data_ptr() + off

    def view(self, off: int, count: int, dtype) -> torch.Tensor:
        esz = torch.empty((), dtype=dtype).element_size()
        return self.buf[off:off + count * esz].view(dtype)


# ---------------------------------------------------------------------------
# engine
# ---------------------------------------------------------------------------
class BatchEngine:
    def __init__(self, max_reqs=1024, max_items=65536, tile_rows=16384, ctas_per_sm=4, stream=None):
        self.L = _bind(N.lib())
        self.stream = stream if stream is not None else torch.cuda.Stream()
        self.max_reqs = max_reqs
        h = ctypes.c_void_p()
        N.check(self.L.ldf_b200_batch_create(max_reqs, max_items, tile_rows, ctas_per_sm,
                                             ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h)))
        self.h = h
        self._rows = (ctypes.c_uint64 * max_reqs)()
        self._ovf = (ctypes.c_int32 * max_reqs)()
        self.event = torch.cuda.Event()

    def submit(self, reqs: list[Request], arena: DeviceArena):
        # inputs and the arena were written on the caller's stream
        self.stream.wait_stream(torch.cuda.current_stream())
        arr = (ldf_batch_request * max(len(reqs), 1))()
        for i, q in enumerate(reqs):
            d = arr[i]
            d.kind, d.vtype, d.n, d.m = q.kind, q.vtype, q.n, q.m
            d.k1, d.v1 = q.k1.data_ptr(), q.v1.data_ptr()
            d.k2 = q.k2.data_ptr() if q.k2 is not None else None
            d.v2 = q.v2.data_ptr() if q.v2 is not None else None
            d.vvalid = q.valid.data_ptr() if q.valid is not None else None
            d.table, d.cap = arena.ptr(q.table_off), q.cap
            base = arena.ptr(q.out_off)
            c = q.out_cap
            d.o0, d.o1, d.o2 = base, base + 8 * c, base + 16 * c
            d.o3 = base + 24 * c if q.kind == JOIN else None
            d.out_cap = c
        N.check(self.L.ldf_b200_batch_run(self.h, arr, len(reqs)))
        self.event.record(self.stream)

    def collect(self, nreq: int):
        N.check(self.L.ldf_b200_batch_wait(self.h, self._rows, self._ovf))
        return [int(self._rows[i]) for i in range(nreq)], [bool(self._ovf[i]) for i in range(nreq)]

    def close(self):
        if self.h:
            self.L.ldf_b200_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


def read_result(q: Request, arena: DeviceArena) -> pa.Table:
    """Copy a completed request's output rows to the host."""
    c, r = q.out_cap, q.rows_out
    base = q.out_off
    k = arena.view(base, c, torch.int64)[:r].cpu().numpy()
    if q.kind == GROUPBY:
        s = arena.view(base + 8 * c, c, torch.float64 if q.vtype == V_FLOAT64 else torch.int64)[:r].cpu().numpy()
        cnt = arena.view(base + 16 * c, c, torch.int64)[:r].cpu().numpy()
        return pa.table({"k": k, "sum": pa.array(s, mask=cnt == 0), "count": cnt})
    lv = arena.view(base + 8 * c, c, torch.int64)[:r].cpu().numpy()
    rk = arena.view(base + 16 * c, c, torch.int64)[:r].cpu().numpy()
    rv = arena.view(base + 24 * c, c, torch.int64)[:r].cpu().numpy()
    return pa.table({"lk": k, "lv": lv, "rk": rk, "rv": rv})


def run_per_op(q: Request) -> pa.Table:
    """The same request through the per-op API (one op per launch sequence)."""
    from legate_dataframe import LogicalColumn, LogicalTable
    from legate_dataframe.lib.groupby_aggregation import groupby_aggregation
    from legate_dataframe.lib.join import JoinType, join

    vt = pa.float64() if q.vtype == V_FLOAT64 else pa.int64()
    if q.kind == GROUPBY:
        v = LogicalColumn.from_torch(q.v1, vt, valid=q.valid)
        t = LogicalTable([LogicalColumn.from_torch(q.k1, pa.int64()), v], ["k", "v"])
        return groupby_aggregation(t, ["k"], [("v", "sum", "sum"), ("v", "count", "count")])
    lt = LogicalTable([LogicalColumn.from_torch(q.k1, pa.int64()), LogicalColumn.from_torch(q.v1, pa.int64())],
                      ["lk", "lv"])
    rt = LogicalTable([LogicalColumn.from_torch(q.k2, pa.int64()), LogicalColumn.from_torch(q.v2, pa.int64())],
                      ["rk", "rv"])
    return join(lt, rt, lhs_keys=["lk"], rhs_keys=["rk"], join_type=JoinType.INNER)


# ---------------------------------------------------------------------------
# admission + continuous batching
# ---------------------------------------------------------------------------
@dataclass
class ServerStats:
    latencies_ms: list = field(default_factory=list)
    rows: int = 0
    requests: int = 0
    batches: int = 0
    fallbacks: int = 0
    wall_s: float = 0.0

    def summary(self) -> dict:
        lat = np.asarray(self.latencies_ms) if self.latencies_ms else np.zeros(1)
        return {
            "requests": self.requests, "batches": self.batches, "fallbacks": self.fallbacks,
            "wall_s": self.wall_s, "req_per_s": self.requests / self.wall_s if self.wall_s else 0.0,
            "rows_per_s": self.rows / self.wall_s if self.wall_s else 0.0,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "max_ms": float(lat.max()),
        }


def admit(queue: deque, arena: DeviceArena, max_reqs: int, max_items: int, tile_rows: int, load_factor: float):
    """Take requests from the head of `queue` (FIFO) while their projected
    hash-table + output bytes fit the arena and the batch capacity; reserve
    their memory.  A head request that does not fit waits (no overtaking)."""
    batch, items = [], 0
    while queue and len(batch) < max_reqs:
        q = queue[0]
        q.plan(load_factor)
        need_items = 2 * (-(-(q.cap + 1) // tile_rows)) + (-(-max(q.n, q.m, 1) // tile_rows)) + 2
        if items + need_items > max_items:
            break
        toff = arena.alloc(q.table_bytes)
        if toff < 0:
            break
        ooff = arena.alloc(q.out_bytes)
        if ooff < 0:
            arena.release(toff, q.table_bytes)
            break
        q.table_off, q.out_off = toff, ooff
        items += need_items
        batch.append(queue.popleft())
    return batch


class Server:
    """Continuous-batching request loop over two engine slots."""

    def __init__(self, arena_bytes=8 << 30, max_reqs=1024, max_items=65536, tile_rows=16384, ctas_per_sm=4,
                 load_factor=0.5, keep_results=False):
        dev = torch.device("cuda", torch.cuda.current_device())
        self.arena = DeviceArena(arena_bytes, dev)
        self.slots = [BatchEngine(max_reqs, max_items, tile_rows, ctas_per_sm) for _ in range(2)]
        self.max_reqs, self.max_items, self.tile_rows = max_reqs, max_items, tile_rows
        self.load_factor = load_factor
        self.keep_results = keep_results

    def _finish(self, slot, batch, stats, t0):
        rows, ovf = slot.collect(len(batch))
        now = time.perf_counter() - t0
        for q, nr, o in zip(batch, rows, ovf):
            q.rows_out = nr
            if o or nr > q.out_cap:
                res = run_per_op(q)  # reservation exceeded: exact per-op path
                torch.cuda.synchronize()
                q.fallback = True
                stats.fallbacks += 1
                q.result = res.to_arrow() if self.keep_results else None
                now = time.perf_counter() - t0
            elif self.keep_results:
                q.result = read_result(q, self.arena)
            q.done = now
            stats.latencies_ms.append(1e3 * (q.done - q.t_in))
            stats.rows += q.rows
            stats.requests += 1
            self.arena.release(q.table_off, q.table_bytes)
            self.arena.release(q.out_off, q.out_bytes)

    def serve(self, requests: list[Request], realtime: bool = True) -> ServerStats:
        """Run `requests` (sorted by arrival, seconds from start).  With
        realtime=False every request is available at t=0 (saturation)."""
        stats = ServerStats()
        pending = deque(sorted(requests, key=lambda q: q.arrival))
        queue: deque = deque()
        running = [None, None]
        t0 = time.perf_counter()
        while pending or queue or any(r is not None for r in running):
            now = time.perf_counter() - t0
            while pending and (not realtime or pending[0].arrival <= now):
                q = pending.popleft()
                q.t_in = q.arrival if realtime else 0.0
                queue.append(q)
            progressed = False
            for i, slot in enumerate(self.slots):
                if running[i] is not None and slot.event.query():
                    self._finish(slot, running[i], stats, t0)
                    running[i] = None
                    progressed = True
            for i, slot in enumerate(self.slots):
                if running[i] is None and queue:
                    batch = admit(queue, self.arena, self.max_reqs, self.max_items, self.tile_rows, self.load_factor)
                    if batch:
                        slot.submit(batch, self.arena)
                        running[i] = batch
                        stats.batches += 1
                        progressed = True
            if not progressed:
                if queue and all(r is None for r in running):
                    # the head request does not fit an empty arena: run it alone per-op
                    q = queue.popleft()
                    res = run_per_op(q)
                    torch.cuda.synchronize()
                    q.result = res.to_arrow() if self.keep_results else None
                    q.done = time.perf_counter() - t0
                    q.fallback = True
                    stats.fallbacks += 1
                    stats.latencies_ms.append(1e3 * (q.done - q.t_in))
                    stats.rows += q.rows
                    stats.requests += 1
                    continue
                time.sleep(20e-6)
        stats.wall_s = time.perf_counter() - t0
        return stats

    def close(self):
        for s in self.slots:
            s.close()


def run_one_op_per_launch(requests: list[Request], realtime: bool = True, keep_results=False) -> ServerStats:
    """Baseline: a serial server running each request through the per-op API."""
    stats = ServerStats()
    t0 = time.perf_counter()
    for q in sorted(requests, key=lambda q: q.arrival):
        arrival = q.arrival if realtime else 0.0
        now = time.perf_counter() - t0
        if realtime and arrival > now:
            time.sleep(arrival - now)
        res = run_per_op(q)
        torch.cuda.synchronize()
        if keep_results:
            q.result = res.to_arrow()
        q.done = time.perf_counter() - t0
        stats.latencies_ms.append(1e3 * (q.done - arrival))
        stats.rows += q.rows
        stats.requests += 1
    stats.wall_s = time.perf_counter() - t0
    return stats


# ---------------------------------------------------------------------------
# autotuner
# ---------------------------------------------------------------------------
class Autotuner:
    """Pick (tile_rows, ctas_per_sm, load_factor) for the batch engine by
    timing one calibration batch per candidate; the choice is persisted per
    GPU name and workload tag."""

    CANDIDATES = [
        (t, c, lf) for t in (4096, 16384, 65536) for c in (2, 4, 8) for lf in (0.35, 0.5)
    ]

    def __init__(self, cache_path: Optional[str] = None):
        default = Path(os.environ.get("LDF_B200_CACHE", Path.home() / ".cache" / "ldf_b200")) / "autotune.json"
        self.path = Path(cache_path) if cache_path else default

    def _load(self) -> dict:
        try:
            return json.loads(self.path.read_text())
        except (OSError, ValueError):
            return {}

    def tune(self, calib: list[Request], tag: str, arena_bytes=4 << 30, candidates=None) -> dict:
        key = f"{torch.cuda.get_device_name()}|{tag}"
        cache = self._load()
        if key in cache:
            return cache[key]
        best = None
        for tile, ctas, lf in candidates or self.CANDIDATES:
            srv = Server(arena_bytes=arena_bytes, tile_rows=tile, ctas_per_sm=ctas, load_factor=lf)
            srv.serve(calib, realtime=False)  # warm
            st = srv.serve(calib, realtime=False)
            srv.close()
            if best is None or st.wall_s < best["wall_s"]:
                best = {"tile_rows": tile, "ctas_per_sm": ctas, "load_factor": lf, "wall_s": st.wall_s}
        cache[key] = best
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            self.path.write_text(json.dumps(cache, indent=1))
        except OSError:
            pass
        return best


# ---------------------------------------------------------------------------
# the served workload: Poisson arrivals, mixed joins and groupbys
# ---------------------------------------------------------------------------
def make_trace(n_requests=8192, rate=2000.0, median_rows=50_000, sigma=1.0, min_rows=1_000, max_rows=20_000_000,
               null_frac=0.1, seed=12, device=None):
    """Requests of the served benchmark: inner join (p=0.5) or int64-key
    groupby SUM/COUNT; rows LogNormal(median, sigma) clipped; keys uniform
    over 0.1 x rows; join payloads int64 uniform on [-2^40, 2^40) (both sides
    `rows` rows), groupby values float64 N(0, 1) with `null_frac` nulls;
    arrivals Poisson at `rate` req/s.  Inputs are generated on the device
    (resident)."""
    rng = np.random.default_rng(seed)
    device = device or torch.device("cuda", torch.cuda.current_device())
    gaps = rng.exponential(1.0 / rate, n_requests)
    arrivals = np.cumsum(gaps) - gaps[0]
    rows = np.clip(np.exp(np.log(median_rows) + sigma * rng.standard_normal(n_requests)), min_rows, max_rows).astype(
        np.int64)
    kinds = rng.random(n_requests) < 0.5
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    reqs = []
    for i in range(n_requests):
        n = int(rows[i])
        kr = max(1, n // 10)
        k1 = torch.randint(0, kr, (n,), device=device, generator=g)
        if kinds[i]:
            v1 = torch.randint(-(2**40), 2**40, (n,), device=device, generator=g)
            k2 = torch.randint(0, kr, (n,), device=device, generator=g)
            v2 = torch.randint(-(2**40), 2**40, (n,), device=device, generator=g)
            reqs.append(Request(JOIN, k1, v1, k2, v2, ndv_hint=kr, arrival=float(arrivals[i]), rid=i))
        else:
            v1 = torch.randn(n, dtype=torch.float64, device=device, generator=g)
            valid = torch.rand(n, device=device, generator=g) >= null_frac
            reqs.append(Request(GROUPBY, k1, v1, valid=valid, ndv_hint=kr, arrival=float(arrivals[i]), rid=i))
    torch.cuda.synchronize(device)
    return reqs
