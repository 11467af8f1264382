"""Parity at the benchmarked sizes themselves: the exact inputs that
``bench.py`` times (``legate_dataframe.workloads``), checked through the C ABI.

* groupby, 200M rows (Zipf(1.1) int64 keys over 10M values, 6.7M groups):
  COUNT(*), COUNT, MIN, MAX and NUNIQUE bit-exact against Acero ``aggregate``
  (the calls of GroupByAggregationTask::cpu_variant, cpp/src/
  groupby_aggregation.cpp:41-94, here with every host thread); SUM and MEAN
  within 1e-12 relative of per-group Neumaier sums (``oracle/neumaier.c``)
  over the group-sorted values.
* joins inner / left / full, 200M probe x 20M build rows: exact row counts,
  null counts per column and order-independent row checksums against the
  join's definition (build keys unique: a probe row matches the build row of
  its key; JoinTask semantics, cpp/src/join.cpp:168-228); and at 20M probe
  rows every row against Acero ``hashjoin`` after a canonical sort.
* 100M string rows: groupby SUM / COUNT(*) against Acero (counts exact, sums
  within 1e-12 of Neumaier); the stable sort (key asc, ts desc) as the exact
  permutation of the input that a stable lexicographic sort gives (ties in
  input order; cpp/src/sort.cpp:324-342); hash_partition(256) bit-exact
  against the oracle's bucket of every row.

The expected permutations and group boundaries are computed with torch's
own sorts on the device (library code, independent of this project's
kernels); the aggregates come from Acero and the C oracle."""

from __future__ import annotations

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest
import torch

pytestmark = pytest.mark.gpu

RTOL = 1e-12
DEV = torch.device("cuda", 0)


def _free():
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def _rel_ok(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    return (x == y) | (np.abs(x - y) <= RTOL * np.maximum(np.abs(y), 1e-300))


# ---------------------------------------------------------------------------
# groupby, 200M rows
# ---------------------------------------------------------------------------
def test_groupby_200m_rows():
    from legate_dataframe import workloads as W
    from legate_dataframe.lib.groupby_aggregation import groupby_aggregation
    from oracle import arrow_ref as A
    from oracle import native

    n = 200_000_000
    keys, v, valid, i = W.zipf_groupby(n, DEV)
    res = groupby_aggregation(W.groupby_table(keys, v, valid, i), ["k"], W.GROUPBY_AGGS).to_arrow()
    res = res.take(pc.sort_indices(res, sort_keys=[("k", "ascending")]))

    # Neumaier sums over the group-sorted rows (torch's stable sort groups them)
    sk, perm = torch.sort(keys, stable=True)
    uniq, counts = torch.unique_consecutive(sk, return_counts=True)
    offsets = np.zeros(uniq.numel() + 1, np.int64)
    np.cumsum(counts.cpu().numpy(), out=offsets[1:])
    sums, vcnt = native.segment_sums(v[perm].cpu().numpy(), valid[perm].cpu().numpy(), offsets)
    del sk, perm, counts
    _free()

    host = pa.table({"k": keys.cpu().numpy(),
                     "v": pa.array(v.cpu().numpy(), mask=valid.cpu().numpy() == 0),
                     "i": i.cpu().numpy()})
    del keys, v, valid, i
    _free()
    ints = [(None, "count_all", "count"), ("v", "count", "count_v"), ("i", "min", "min_i"),
            ("i", "max", "max_i"), ("i", "count_distinct", "nunique_i")]
    exp = A.groupby(host, ["k"], ints, use_threads=True)
    del host
    exp = exp.take(pc.sort_indices(exp, sort_keys=[("k", "ascending")]))

    assert res.num_rows == exp.num_rows == uniq.numel()
    assert res.column("k").equals(exp.column("k"))
    assert np.array_equal(res.column("k").to_numpy(), uniq.cpu().numpy())
    for name in ("count", "count_v", "min_i", "max_i", "nunique_i"):
        assert res.column(name).equals(exp.column(name)), name
    assert np.array_equal(res.column("count_v").to_numpy(), vcnt)
    has = vcnt > 0
    for name, want in (("sum_v", sums), ("mean_v", sums / np.maximum(vcnt, 1))):
        col = res.column(name).combine_chunks()
        assert np.array_equal(np.asarray(col.is_valid()), has), name
        got = col.fill_null(0).to_numpy()[has]
        ok = _rel_ok(got, want[has])
        assert ok.all(), f"{name}: {int((~ok).sum())} groups beyond {RTOL}"
    _free()


# ---------------------------------------------------------------------------
# joins, 200M probe x 20M build rows
# ---------------------------------------------------------------------------
_C1 = 0xFF51AFD7ED558CCD - (1 << 64)
_C2 = 0xC4CEB9FE1A85EC53 - (1 << 64)


def _mix(x: torch.Tensor) -> torch.Tensor:
    """MurmurHash3 fmix64 on int64 tensors (logical shifts, wrapping products)."""
    m31 = (1 << 31) - 1
    x = x ^ ((x >> 33) & m31)
    x = x * _C1
    x = x ^ ((x >> 33) & m31)
    x = x * _C2
    return x ^ ((x >> 33) & m31)


def _col_bits(c) -> tuple[torch.Tensor, torch.Tensor]:
    """(int64 value bits, bool validity) of a fixed-width device column."""
    from legate_dataframe import _native as N

    n = c.size
    w = N.TYPE_WIDTH[c.ldf_type]
    raw = c.data[: n * w]
    bits = {1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}[w]
    x = raw.view(bits).to(torch.int64)
    ok = c.valid[:n].bool() if c.valid is not None else torch.ones(n, dtype=torch.bool, device=raw.device)
    return x, ok


def _row_checksum(cols) -> tuple[int, ...]:
    """Order-independent checksum of a table's rows: every row hashes its
    columns' (value, valid) pairs together, and the row hashes are summed
    (two different mixes, each as two 32-bit halves, so no sum overflows)."""
    h1 = None
    h2 = None
    for j, (x, ok) in enumerate(cols):
        a = torch.where(ok, _mix(x + (j + 1) * 0x9E3779B9), torch.full_like(x, 0x5BD1E995 + j))
        b = torch.where(ok, _mix(x ^ ((j + 7) * 0x2545F491)), torch.full_like(x, 0x27D4EB2F + j))
        h1 = a if h1 is None else _mix(h1 + a)
        h2 = b if h2 is None else h2 + b
    m = 0xFFFFFFFF
    return tuple(int(t.sum()) for t in (h1 & m, (h1 >> 32) & m, h2 & m, (h2 >> 32) & m))


def _expected_join_cols(J, how: str):
    nb = J.bkey.numel()
    inv = torch.empty(nb, dtype=torch.int64, device=DEV)
    inv[J.bkey.long()] = torch.arange(nb, device=DEV)
    inrange = J.pvalid & (J.pkey >= 0) & (J.pkey < nb)
    brow = torch.where(inrange, inv[J.pkey.long().clamp(0, nb - 1)], torch.full_like(inv[:1], -1))
    matched = brow >= 0
    lk = J.pkey.to(torch.int64)
    lv = J.ppay.view(torch.int64)
    ones = torch.ones_like(matched)
    safe = brow.clamp(min=0)
    rk, r1, r2 = J.bkey[safe].to(torch.int64), J.bp1[safe], J.bp2[safe]
    if how == "inner":
        return [(lk[matched], ones[matched]), (lv[matched], ones[matched]), (rk[matched], ones[matched]),
                (r1[matched], ones[matched]), (r2[matched], ones[matched])]
    cols = [(lk, J.pvalid), (lv, ones), (rk, matched), (r1, matched), (r2, matched)]
    if how == "left":
        return cols
    hit = torch.zeros(nb, dtype=torch.bool, device=DEV)
    hit[brow[matched]] = True
    un = torch.nonzero(~hit).squeeze(1)
    z = torch.zeros(un.numel(), dtype=torch.int64, device=DEV)
    f = torch.zeros(un.numel(), dtype=torch.bool, device=DEV)
    t = torch.ones(un.numel(), dtype=torch.bool, device=DEV)
    tail = [(z, f), (z, f), (J.bkey[un].to(torch.int64), t), (J.bp1[un], t), (J.bp2[un], t)]
    return [(torch.cat([a, b]), torch.cat([m, mb])) for (a, m), (b, mb) in zip(cols, tail)]


@pytest.mark.parametrize("how", ["inner", "left", "full"])
def test_join_200m_x_20m(how):
    from legate_dataframe import workloads as W
    from legate_dataframe.lib.join import JoinType, join

    J = W.int32_join(200_000_000, 20_000_000, DEV)
    lt, rt = J.tables()
    res = join(lt, rt, lhs_keys=["lk"], rhs_keys=["rk"], join_type=JoinType[how.upper()])
    assert res.get_column_names() == ["lk", "lv", "rk", "r1", "r2"]
    got = [_col_bits(c) for c in res.get_columns()]
    exp = _expected_join_cols(J, how)
    assert got[0][0].numel() == exp[0][0].numel(), "row count"
    for j, ((_, a), (_, b)) in enumerate(zip(got, exp)):
        assert int(a.sum()) == int(b.sum()), f"valid count of column {j}"
    assert _row_checksum(got) == _row_checksum(exp)
    del res, got, exp, lt, rt, J
    _free()


def _lexsort_rows(cols) -> list[torch.Tensor]:
    """The rows of (bits, valid) columns in lexicographic order (nulls
    first), by stable sorts from the last column to the first."""
    n = cols[0][0].numel()
    order = torch.arange(n, device=DEV)
    for x, ok in reversed(cols):
        key = torch.where(ok, x, torch.zeros_like(x))[order]
        order = order[torch.sort(key, stable=True).indices]
        order = order[torch.sort(ok[order].to(torch.int8), stable=True).indices]
    return [torch.where(ok, x, torch.zeros_like(x))[order] for x, ok in cols] + [c[1][order] for c in cols]


def _arrow_bits(t: pa.Table):
    out = []
    for c in t.columns:
        a = c.combine_chunks()
        ok = np.asarray(a.is_valid())
        vals = a.fill_null(0).to_numpy(zero_copy_only=False)
        if vals.dtype.kind == "f":
            vals = vals.view(np.int64 if vals.dtype.itemsize == 8 else np.int32)
        out.append((torch.from_numpy(vals.astype(np.int64)).to(DEV), torch.from_numpy(ok).to(DEV)))
    return out


@pytest.mark.parametrize("how", ["inner", "left", "full"])
def test_join_20m_x_20m_rows_vs_acero(how):
    """Every output row, at 20M probe rows against the full 20M-row build."""
    from legate_dataframe import workloads as W
    from legate_dataframe.lib.join import JoinType, join
    from oracle import arrow_ref as A

    J = W.int32_join(20_000_000, 20_000_000, DEV)
    lt, rt = J.tables()
    res = join(lt, rt, lhs_keys=["lk"], rhs_keys=["rk"], join_type=JoinType[how.upper()])
    got = _lexsort_rows([_col_bits(c) for c in res.get_columns()])
    lh = pa.table({"lk": pa.array(J.pkey.cpu().numpy(), mask=~J.pvalid.cpu().numpy()), "lv": J.ppay.cpu().numpy()})
    rh = pa.table({"rk": J.bkey.cpu().numpy(), "r1": J.bp1.cpu().numpy(), "r2": J.bp2.cpu().numpy()})
    exp_t = A.join(lh, rh, ["lk"], ["rk"], how, True, use_threads=True)
    assert exp_t.column_names == ["lk", "lv", "rk", "r1", "r2"]
    exp = _lexsort_rows(_arrow_bits(exp_t))
    assert got[0].numel() == exp[0].numel()
    for j, (a, b) in enumerate(zip(got, exp)):
        assert torch.equal(a, b), f"column part {j} differs"
    del res, got, exp, J, lt, rt
    _free()


# ---------------------------------------------------------------------------
# 100M string rows: groupby, stable sort, hash_partition
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def strings_100m():
    from legate_dataframe import workloads as W

    S = W.string_rows(100_000_000, DEV)
    d = S.dictionary()
    assert len(set(d)) == len(d), "dictionary strings are distinct"
    yield S, d
    del S
    _free()


def _dict_rank(d: list[bytes]) -> torch.Tensor:
    order = sorted(range(len(d)), key=d.__getitem__)
    rank = np.empty(len(d), np.int64)
    rank[np.asarray(order)] = np.arange(len(d))
    return torch.from_numpy(rank).to(DEV)


def _assert_permuted(out, S, perm: torch.Tensor, chunk: int = 20_000_000):
    """`out` (k, ts, v) equals the input rows taken in the order `perm`."""
    k, ts, v = out.get_columns()
    n = perm.numel()
    assert k.size == ts.size == v.size == n
    assert torch.equal(ts.data[: 8 * n].view(torch.int64), S.ts[perm])
    assert torch.equal(v.data[: 4 * n].view(torch.int32), S.val.view(torch.int32)[perm])
    rng = k.data[: 16 * n].view(torch.int64).view(n, 2)
    dlen = S.d_off[1:] - S.d_off[:-1]
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        p = S.pick[perm[s:e]]
        want_len = dlen[p]
        lo = rng[s:e, 0] - k.chars_base
        ln = rng[s:e, 1] - rng[s:e, 0] + 1
        assert torch.equal(ln, want_len), "string lengths"
        tot = int(ln.sum())
        start = torch.cumsum(ln, 0) - ln
        row = torch.repeat_interleave(torch.arange(e - s, device=DEV), ln)
        pos = torch.arange(tot, device=DEV) - start[row]
        assert torch.equal(k.chars[lo[row] + pos], S.d_chars[S.d_off[p][row] + pos]), "string characters"
        del p, lo, ln, start, row, pos


def test_strings_100m_groupby(strings_100m):
    from legate_dataframe.lib.groupby_aggregation import groupby_aggregation
    from oracle import arrow_ref as A
    from oracle import native

    S, d = strings_100m
    res = groupby_aggregation(S.table(), ["k"], [("v", "sum", "s"), (None, "count_all", "c")]).to_arrow()
    res = res.take(pc.sort_indices(res, sort_keys=[("k", "ascending")]))
    pick = S.pick.cpu().numpy()
    dictionary = pa.array(d, pa.binary()).cast(pa.string())
    host = pa.table({"k": pa.DictionaryArray.from_arrays(pa.array(pick.astype(np.int32)), dictionary)
                     .cast(pa.string()), "v": S.val.cpu().numpy()})
    exp = A.groupby(host, ["k"], [(None, "count_all", "c")], use_threads=True)
    del host
    exp = exp.take(pc.sort_indices(exp, sort_keys=[("k", "ascending")]))
    assert res.num_rows == exp.num_rows
    assert res.column("k").equals(exp.column("k"))
    assert res.column("c").equals(exp.column("c"))
    # Neumaier sums per dictionary entry, ordered like the sorted keys
    sp, perm = torch.sort(S.pick, stable=True)
    up, cnt = torch.unique_consecutive(sp, return_counts=True)
    off = np.zeros(up.numel() + 1, np.int64)
    np.cumsum(cnt.cpu().numpy(), out=off[1:])
    sums, _ = native.segment_sums(S.val[perm].cpu().numpy(), None, off)
    rank = _dict_rank(d)[up].cpu().numpy()
    want = sums[np.argsort(rank)]
    got = res.column("s").to_numpy()
    ok = _rel_ok(got, want)
    assert ok.all(), f"{int((~ok).sum())} group sums beyond {RTOL}"
    del sp, perm, up, cnt
    _free()


def test_strings_100m_stable_sort(strings_100m):
    from legate_dataframe.lib.sort import sort

    S, d = strings_100m
    out = sort(S.table(), ["k", "ts"], sort_ascending=[True, False], stable=True)
    rk = _dict_rank(d)[S.pick]
    p1 = torch.sort(S.ts, descending=True, stable=True).indices
    perm = p1[torch.sort(rk[p1], stable=True).indices]
    del rk, p1
    _assert_permuted(out, S, perm)
    del out, perm
    _free()


def test_strings_100m_hash_partition(strings_100m):
    from legate_dataframe.lib.hash_partition import hash_partition
    from oracle import relational as R

    S, d = strings_100m
    out, offsets = hash_partition(S.table(), ["k"], 256)
    hv = R.string_hashes(S.d_chars.cpu().numpy(), S.d_off.cpu().numpy())
    seed = np.full(len(hv), 0x243F6A8885A308D3, dtype=np.uint64)
    bucket_d = (R._hash_combine(seed, hv) % np.uint64(256)).astype(np.int64)
    bucket = torch.from_numpy(bucket_d).to(DEV)[S.pick]
    perm = torch.sort(bucket, stable=True).indices
    want = np.zeros(257, np.int64)
    np.cumsum(torch.bincount(bucket, minlength=256).cpu().numpy(), out=want[1:])
    assert list(offsets) == want.tolist()
    del bucket
    _assert_permuted(out, S, perm)
    del out, perm
    _free()
