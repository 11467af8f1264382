"""Seeded synthetic inputs of the benchmark workloads, generated on the device.

The reference measures on no public dataset; these generators reproduce the
shapes, sizes and value distributions of its benchmark configurations
(``python/benchmarks/join.py`` defines the join one; the others are this
project's groupby / join / string workloads).  ``bench.py`` times the ops on
them and the full-size parity tests check the ops on the very same inputs.

* ``zipf_groupby``: int64 keys Zipf(s=1.1) over 10M distinct values,
  float64 N(0,1) with 10% nulls, int32 U[0, 1e6).
* ``int32_join``: build side of unique int32 keys (a permutation of
  [0, n_build)) with two int64 payloads; probe side whose int32 keys hit a
  build key of Zipf(0.9) rank with probability 0.8 and otherwise fall on
  [n_build, 2 n_build), 5% null keys, one float64 payload U(0,1).
* ``string_rows``: string keys drawn Zipf(1.0) from a 2M-entry dictionary
  of [a-z0-9] strings of length U{8..24}; int64 timestamps over one year in
  microseconds; float32 LogNormal(0,1) values.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import pyarrow as pa
import torch

GROUPBY_KEYS = 10_000_000
GROUPBY_AGGS = [
    ("v", "sum", "sum_v"),
    ("v", "mean", "mean_v"),
    (None, "count_all", "count"),
    ("v", "count", "count_v"),
    ("i", "min", "min_i"),
    ("i", "max", "max_i"),
    ("i", "count_distinct", "nunique_i"),
]
STRING_DICT = 2_000_000
TS0 = 1_600_000_000_000_000
TS_SPAN = 365 * 86400 * 10**6


def _zipf_cdf(n: int, s: float, device) -> torch.Tensor:
    cdf = torch.cumsum(torch.arange(1, n + 1, device=device, dtype=torch.float64).pow(-s), 0)
    cdf /= cdf[-1].clone()
    return cdf


def zipf_groupby(n_rows: int, device):
    """(keys int64, v float64, valid uint8, i int32) of the groupby workload."""
    g = torch.Generator(device=device)
    cdf = _zipf_cdf(GROUPBY_KEYS, 1.1, device)
    g.manual_seed(3)
    perm = torch.randperm(GROUPBY_KEYS, device=device, generator=g)
    key_values = perm.to(torch.int64) * 2_654_435_761 + 12_345  # 10M distinct int64 values
    keys = torch.empty(n_rows, dtype=torch.int64, device=device)
    g.manual_seed(1)
    chunk = 50_000_000
    for s in range(0, n_rows, chunk):
        e = min(n_rows, s + chunk)
        u = torch.rand(e - s, dtype=torch.float64, device=device, generator=g)
        r = torch.searchsorted(cdf, u).clamp_(max=GROUPBY_KEYS - 1)
        keys[s:e] = key_values[r]
        del u, r
    del cdf, perm
    g.manual_seed(4)
    v = torch.randn(n_rows, dtype=torch.float64, device=device, generator=g)
    valid = (torch.rand(n_rows, device=device, generator=g) >= 0.10).to(torch.uint8)
    g.manual_seed(5)
    i = torch.randint(0, 1_000_000, (n_rows,), dtype=torch.int32, device=device, generator=g)
    torch.cuda.synchronize(device)
    return keys, v, valid, i


def groupby_table(keys, v, valid, i):
    from legate_dataframe import LogicalColumn, LogicalTable

    return LogicalTable([LogicalColumn.from_torch(keys, pa.int64()),
                         LogicalColumn.from_torch(v, pa.float64(), valid),
                         LogicalColumn.from_torch(i, pa.int32())], ["k", "v", "i"])


@dataclass
class JoinInputs:
    bkey: torch.Tensor   # int32 [n_build], a permutation of [0, n_build)
    bp1: torch.Tensor    # int64 [n_build]
    bp2: torch.Tensor    # int64 [n_build]
    pkey: torch.Tensor   # int32 [n_probe]
    pvalid: torch.Tensor  # bool [n_probe]
    ppay: torch.Tensor   # float64 [n_probe]

    def tables(self):
        from legate_dataframe import LogicalColumn, LogicalTable

        lt = LogicalTable([LogicalColumn.from_torch(self.pkey, pa.int32(), valid=self.pvalid),
                           LogicalColumn.from_torch(self.ppay, pa.float64())], ["lk", "lv"])
        rt = LogicalTable([LogicalColumn.from_torch(self.bkey, pa.int32()),
                           LogicalColumn.from_torch(self.bp1, pa.int64()),
                           LogicalColumn.from_torch(self.bp2, pa.int64())], ["rk", "r1", "r2"])
        return lt, rt


def int32_join(n_probe: int, n_build: int, device) -> JoinInputs:
    g = torch.Generator(device=device)
    g.manual_seed(6)
    bkey = torch.randperm(n_build, device=device, generator=g).to(torch.int32)
    bp1 = torch.randint(-(2**40), 2**40, (n_build,), device=device, generator=g)
    bp2 = torch.randint(-(2**40), 2**40, (n_build,), device=device, generator=g)
    g.manual_seed(7)
    cdf = _zipf_cdf(n_build, 0.9, device)
    u = torch.rand(n_probe, device=device, generator=g, dtype=torch.float64)
    hit = torch.rand(n_probe, device=device, generator=g) < 0.8
    idx = torch.searchsorted(cdf, u).clamp_(max=n_build - 1)
    miss = torch.randint(n_build, 2 * n_build, (n_probe,), device=device, generator=g, dtype=torch.int32)
    pkey = torch.where(hit, bkey[idx], miss)
    pvalid = torch.rand(n_probe, device=device, generator=g) >= 0.05
    ppay = torch.rand(n_probe, device=device, generator=g, dtype=torch.float64)
    del cdf, u, hit, idx, miss
    torch.cuda.synchronize(device)
    return JoinInputs(bkey, bp1, bp2, pkey, pvalid, ppay)


@dataclass
class StringInputs:
    pick: torch.Tensor     # int64 [n] dictionary index of each row's key
    ranges: torch.Tensor   # int64 [n, 2] inclusive char ranges (legate Rect<1>)
    chars: torch.Tensor    # uint8 characters of the rows, in row order
    ts: torch.Tensor       # int64 [n] timestamps (us)
    val: torch.Tensor      # float32 [n]
    d_chars: torch.Tensor  # uint8 characters of the dictionary
    d_off: torch.Tensor    # int64 [STRING_DICT + 1] dictionary offsets

    def table(self):
        from legate_dataframe import LogicalColumn, LogicalTable
        from legate_dataframe import _native as N

        n = self.ts.numel()
        key = LogicalColumn(pa.string(), N.LDF_STRING, n, self.ranges.view(torch.uint8).reshape(-1), None,
                            chars=self.chars, chars_base=0, num_chars=self.chars.numel())
        return LogicalTable([key, LogicalColumn.from_torch(self.ts, pa.timestamp("us")),
                             LogicalColumn.from_torch(self.val, pa.float32())], ["k", "ts", "v"])

    def dictionary(self) -> list[bytes]:
        dc = self.d_chars.cpu().numpy().tobytes()
        do = self.d_off.cpu().numpy()
        return [dc[do[j]:do[j + 1]] for j in range(len(do) - 1)]


def string_rows(n: int, device) -> StringInputs:
    rng = np.random.default_rng(9)
    lens = rng.integers(8, 25, STRING_DICT)
    alphabet = np.frombuffer(b"abcdefghijklmnopqrstuvwxyz0123456789", dtype=np.uint8)
    d_chars = torch.from_numpy(alphabet[rng.integers(0, 36, int(lens.sum()))].copy()).to(device)
    doff = np.zeros(STRING_DICT + 1, np.int64)
    np.cumsum(lens, out=doff[1:])
    d_off = torch.from_numpy(doff).to(device)
    g = torch.Generator(device=device)
    g.manual_seed(9)
    cdf = _zipf_cdf(STRING_DICT, 1.0, device)
    pick = torch.searchsorted(cdf, torch.rand(n, device=device, generator=g, dtype=torch.float64))
    pick = pick.clamp_(max=STRING_DICT - 1)
    row_len = (d_off[1:] - d_off[:-1])[pick]
    row_off = torch.cumsum(row_len, 0) - row_len
    rowid = torch.repeat_interleave(torch.arange(n, device=device), row_len)
    pos = torch.arange(int(row_len.sum()), device=device)
    chars = d_chars[d_off[pick][rowid] + (pos - row_off[rowid])]
    del rowid, pos, cdf
    ranges = torch.stack([row_off, row_off + row_len - 1], 1).contiguous()
    ts = torch.randint(TS0, TS0 + TS_SPAN, (n,), device=device, generator=g)
    val = torch.exp(torch.randn(n, device=device, generator=g)).to(torch.float32)
    torch.cuda.synchronize(device)
    return StringInputs(pick, ranges, chars, ts, val, d_chars, d_off)
