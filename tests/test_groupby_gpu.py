"""Parity of the sm_100a hash groupby (through the C ABI) with the oracle and
golden vectors: every supported aggregation and count mode, int/float/string
and multi-column keys, null keys and values, skewed (Zipf) keys that exercise
the shared-memory pre-aggregation, the sampled-estimate path and overflow
retry.  Integer aggregates and NUNIQUE bit-exact; float SUM/MEAN within 1e-12
relative of the Neumaier oracle."""

import zlib

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

from ldf_testing import agg_spec, assert_tables_equal, load_golden
from oracle import relational as R

pytestmark = pytest.mark.gpu

RTOL = 1e-12
GB_CASES = [c for c in load_golden() if c["op"] == "groupby"]


def run_groupby(table, keys, aggs):
    from legate_dataframe import LogicalTable
    from legate_dataframe.lib.groupby_aggregation import groupby_aggregation

    return groupby_aggregation(LogicalTable.from_arrow(table), keys, aggs).to_arrow()


@pytest.mark.parametrize("case", GB_CASES, ids=[c["name"] for c in GB_CASES])
def test_groupby_golden(case):
    t = case["tables"]
    res = run_groupby(t["table"], case["keys"], agg_spec(case["aggs"]))
    # golden expectations come from Arrow's own (uncompensated) float sums
    assert_tables_equal(res, t["expected"], sort_by=case["keys"], rtol=1e-12)


ALL_AGGS = [
    ("v", "sum", "sum"), ("v", "mean", "mean"), ("v", "count", "count"), (None, "count_all", "count_all"),
    ("i", "min", "min"), ("i", "max", "max"), ("i", "count_distinct", "nunique"), ("i", "sum", "isum"),
    ("v", "min", "vmin"), ("v", "max", "vmax"), ("i", "mean", "imean"),
    ("v", ("count", pc.CountOptions(mode="all")), "c_all"),
    ("v", ("count", pc.CountOptions(mode="only_null")), "c_null"),
    ("v", ("count_distinct", pc.CountOptions(mode="all")), "nd_all"),
]


def _table(rng, n, key_kind, ngroups, key_null_p=0.02, zipf=None):
    if zipf:
        ranks = np.minimum(rng.zipf(zipf, n), ngroups) - 1
        perm = rng.permutation(ngroups)
        raw = perm[ranks]
    else:
        raw = rng.integers(0, ngroups, n)
    kmask = rng.random(n) < key_null_p if key_null_p else None
    if key_kind == "string":
        k = pa.array([None if (kmask is not None and m) else f"g{x}" for x, m in
                      zip(raw, kmask if kmask is not None else np.zeros(n, bool))], pa.string())
    else:
        k = pa.array(raw.astype(key_kind), mask=kmask)
    v = pa.array(rng.normal(size=n), mask=rng.random(n) < 0.1)
    i = pa.array(rng.integers(0, 1000, n).astype(np.int32))
    return pa.table({"k": k, "v": v, "i": i})


@pytest.mark.parametrize("key_kind", ["int32", "int64", "float64", "string", "int8"])
def test_groupby_all_aggs(key_kind):
    rng = np.random.default_rng(17)
    t = _table(rng, 20000, key_kind, 120 if key_kind != "int8" else 100)
    res = run_groupby(t, ["k"], ALL_AGGS)
    exp = R.groupby(t, ["k"], ALL_AGGS)
    assert_tables_equal(res, exp, sort_by=["k"], rtol=RTOL)


def test_groupby_multikey_nulls():
    rng = np.random.default_rng(23)
    n = 30000
    t = pa.table({
        "a": pa.array(rng.integers(0, 7, n).astype(np.int32), mask=rng.random(n) < 0.05),
        "b": pa.array([None if m else f"s{x}" for x, m in zip(rng.integers(0, 9, n), rng.random(n) < 0.05)]),
        "v": pa.array(rng.normal(size=n) * 1e3, mask=rng.random(n) < 0.2),
        "i": pa.array(rng.integers(-50, 50, n).astype(np.int64), mask=rng.random(n) < 0.1),
    })
    aggs = [("v", "sum", "s"), ("v", "mean", "m"), ("i", "min", "mn"), ("i", "max", "mx"),
            ("i", "count_distinct", "nd"), ("i", ("count_distinct", pc.CountOptions(mode="all")), "nda"),
            (None, "count_all", "n"), ("i", "sum", "is")]
    res = run_groupby(t, ["a", "b"], aggs)
    exp = R.groupby(t, ["a", "b"], aggs)
    assert_tables_equal(res, exp, sort_by=["a", "b"], rtol=RTOL)


@pytest.mark.parametrize("n,ngroups", [(200_000, 50_000), (2_000_000, 300_000)])
def test_groupby_zipf_large(n, ngroups):
    # skewed keys (heavy hitters in shared memory) and the sampled estimate
    rng = np.random.default_rng(n)
    t = _table(rng, n, "int64", ngroups, key_null_p=0.0, zipf=1.1)
    aggs = [("v", "sum", "sum"), ("v", "mean", "mean"), (None, "count_all", "n"), ("v", "count", "c"),
            ("i", "min", "mn"), ("i", "max", "mx"), ("i", "count_distinct", "nd")]
    res = run_groupby(t, ["k"], aggs)
    exp = R.groupby(t, ["k"], aggs)
    assert_tables_equal(res, exp, sort_by=["k"], rtol=RTOL)


def test_groupby_float_sum_cancellation():
    # sums near zero: the fixed-point accumulator is exact, the Neumaier
    # oracle nearly so; plain fp64 atomics would miss 1e-12 here
    rng = np.random.default_rng(5)
    n = 400_000
    g = rng.integers(0, 1000, n)
    x = rng.normal(size=n) * 1e6
    x = np.concatenate([x, -x])
    g = np.concatenate([g, g])
    x[::7] += rng.normal(size=len(x[::7]))
    t = pa.table({"k": g.astype(np.int64), "v": x})
    res = run_groupby(t, ["k"], [("v", "sum", "s")])
    exp = R.groupby(t, ["k"], [("v", "sum", "s")])
    assert_tables_equal(res, exp, sort_by=["k"], rtol=RTOL)


def test_groupby_special_floats():
    t = pa.table({"k": pa.array([1, 1, 2, 2, 3, 3, 4, 5, 5], pa.int64()),
                  "v": pa.array([1.0, np.nan, np.inf, 1.0, np.inf, -np.inf, 1e-300, 1e300, 1e300])})
    res = run_groupby(t, ["k"], [("v", "sum", "s"), ("v", "mean", "m")]).to_pydict()
    order = np.argsort(res["k"])
    s = np.array(res["s"])[order]
    assert np.isnan(s[0]) and s[1] == np.inf and np.isnan(s[2]) and s[3] == 1e-300 and s[4] == 2e300


def test_groupby_deterministic_bits():
    rng = np.random.default_rng(99)
    t = _table(rng, 500_000, "int64", 20_000, zipf=1.05)
    aggs = [("v", "sum", "s"), ("v", "mean", "m")]
    a = run_groupby(t, ["k"], aggs).sort_by("k")
    b = run_groupby(t, ["k"], aggs).sort_by("k")
    assert a.equals(b)


def test_groupby_empty_and_single():
    e = pa.table({"k": pa.array([], pa.int64()), "v": pa.array([], pa.float64())})
    res = run_groupby(e, ["k"], [("v", "sum", "s"), (None, "count_all", "n")])
    assert res.num_rows == 0
    one = pa.table({"k": pa.array([None], pa.int64()), "v": pa.array([None], pa.float64())})
    res = run_groupby(one, ["k"], [("v", "sum", "s"), (None, "count_all", "n"), ("v", "count", "c")])
    assert res.to_pydict() == {"k": [None], "s": [None], "n": [1], "c": [0]}


def test_groupby_sentinel_key_value():
    # the 8-byte key equal to the table's empty marker takes the extra slot
    sentinel = np.int64(np.uint64(0x7FF4DEAD7FF4BEEF).view(np.int64))
    t = pa.table({"k": pa.array([sentinel, 1, sentinel, None, 1], pa.int64()), "v": [1.0, 2.0, 3.0, 4.0, 5.0]})
    res = run_groupby(t, ["k"], [("v", "sum", "s")])
    exp = R.groupby(t, ["k"], [("v", "sum", "s")])
    assert_tables_equal(res, exp, sort_by=["k"])


@pytest.mark.parametrize("vkind", ["int32_neg", "int32_wide", "int8", "int16", "uint32", "uint8", "float32", "bool"])
@pytest.mark.parametrize("budget_mb", [None, "0", "1"])
def test_groupby_nunique_value_kinds(vkind, budget_mb, monkeypatch):
    # NUNIQUE through the value bitmaps of frequent ranks (small value ranges,
    # any budget) and through the pair set (wide ranges, budget 0)
    if budget_mb is not None:
        monkeypatch.setenv("LDF_B200_ND_BITMAP_MB", budget_mb)
    rng = np.random.default_rng(31)
    n = 300_000
    ranks = np.minimum(rng.zipf(1.2, n), 5000) - 1
    k = rng.permutation(5000)[ranks].astype(np.int64)
    if vkind == "int32_neg":
        v = pa.array(rng.integers(-3000, 2000, n).astype(np.int32), mask=rng.random(n) < 0.1)
    elif vkind == "int32_wide":
        v = pa.array(rng.integers(-2**31, 2**31 - 1, n).astype(np.int32))
    elif vkind == "int8":
        v = pa.array(rng.integers(-128, 128, n).astype(np.int8), mask=rng.random(n) < 0.05)
    elif vkind == "int16":
        v = pa.array(rng.integers(-30000, 30000, n).astype(np.int16))
    elif vkind == "uint32":
        v = pa.array(rng.integers(4_000_000_000, 4_000_100_000, n).astype(np.uint32))
    elif vkind == "uint8":
        v = pa.array(rng.integers(0, 256, n).astype(np.uint8))
    elif vkind == "float32":
        x = rng.integers(-500, 500, n).astype(np.float32) / 4
        x[::97] = -0.0
        x[::89] = np.nan
        v = pa.array(x)
    else:
        v = pa.array(rng.random(n) < 0.3, mask=rng.random(n) < 0.1)
    t = pa.table({"k": k, "v": v})
    aggs = [("v", "count_distinct", "nd"), ("v", ("count_distinct", pc.CountOptions(mode="all")), "nda")]
    res = run_groupby(t, ["k"], aggs)
    exp = R.groupby(t, ["k"], aggs)
    assert_tables_equal(res, exp, sort_by=["k"])


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_groupby_special_float_keys_by_bits(dtype):
    from ldf_testing import special_float_tables

    t, _, _ = special_float_tables(dtype)
    aggs = [("v", "sum", "s"), ("w", "count_distinct", "nd"), (None, "count_all", "n")]
    res = run_groupby(t, ["k"], aggs)
    exp = R.groupby(t, ["k"], aggs)
    assert res.num_rows == 5
    assert_tables_equal(res, exp, sort_by=["s"])


@pytest.mark.parametrize("segments", ["1", "0"])
@pytest.mark.parametrize("vtype", [np.int32, np.uint32])
def test_groupby_nunique_size_tiers(segments, vtype, monkeypatch):
    # group sizes on both sides of every tier boundary of the per-rank
    # segments (8192 / 512 / 16 rows), a 32-bit-wide value range (no value
    # bitmaps), the all-ones bit pattern as a value, and null values
    monkeypatch.setenv("LDF_B200_ND_SEGMENTS", segments)
    rng = np.random.default_rng(77)
    sizes = ([40000, 16385, 16384, 9000, 8193, 8192, 5000, 513, 512, 511, 300, 17, 16, 15, 10, 2, 1]
             + [1] * 2000 + [3] * 1000 + [40] * 500 + [700] * 40)
    keys = np.repeat(np.arange(len(sizes), dtype=np.int64) * 7 + 3, sizes)
    vals = np.empty(len(keys), dtype=np.int64)
    pos = 0
    for s in sizes:
        base = int(rng.integers(0, 2**32))
        vals[pos:pos + s] = (base + rng.integers(0, max(2, s // 2), s) * 2654435761) % 2**32
        pos += s
    vals[rng.random(len(vals)) < 0.01] = 2**32 - 1
    v = vals.astype(np.uint32).view(vtype)
    perm = rng.permutation(len(keys))
    t = pa.table({"k": keys[perm], "v": pa.array(v[perm], mask=rng.random(len(keys)) < 0.1)})
    aggs = [("v", "count_distinct", "nd"), ("v", ("count_distinct", pc.CountOptions(mode="all")), "nda"),
            (None, "count_all", "n")]
    res = run_groupby(t, ["k"], aggs)
    exp = R.groupby(t, ["k"], aggs)
    assert_tables_equal(res, exp, sort_by=["k"])


def _on_host(col, pinned):
    """The same column with every buffer in host memory (pinned or pageable)."""
    from legate_dataframe import LogicalColumn

    def h(t):
        if t is None:
            return None
        t = t.cpu()
        return t.pin_memory() if pinned else t

    return LogicalColumn(col.arrow_type, col.ldf_type, col.size, h(col.data), h(col.valid), h(col.chars),
                         col.chars_base, col.num_chars)


@pytest.mark.parametrize("key_kind", ["int64", "string", "int32"])
@pytest.mark.parametrize("pinned", [True, False])
def test_groupby_host_resident_inputs(key_kind, pinned):
    """Input columns in host memory are copied to the device inside the op
    (overlapped with its passes); the result is bit-identical to the one of
    the same columns resident on the device, on two calls in a row."""
    from legate_dataframe import LogicalTable
    from legate_dataframe.lib.groupby_aggregation import groupby_aggregation

    rng = np.random.default_rng(23)
    t = _table(rng, 200_000, key_kind, 3000, zipf=1.2)
    dev = LogicalTable.from_arrow(t)
    host = LogicalTable([_on_host(c, pinned) for c in dev.get_columns()], dev.get_column_names())
    exp = groupby_aggregation(dev, ["k"], ALL_AGGS).to_arrow()
    for _ in range(2):
        res = groupby_aggregation(host, ["k"], ALL_AGGS).to_arrow()
        assert_tables_equal(res, exp, sort_by=["k"])


@pytest.mark.parametrize("vkind", ["int32_neg", "int8", "int16", "uint8", "uint32", "bool"])
@pytest.mark.parametrize("other", [False, True])
def test_groupby_nunique_with_min_max(vkind, other):
    """MIN / MAX / COUNT beside NUNIQUE on one column, with and without
    another aggregated column; ranks below and above the shared-memory hot
    limits of the column and NUNIQUE kernels are both present."""
    rng = np.random.default_rng(zlib.crc32(f"{vkind}{other}".encode()))
    n = 400_000
    ranks = np.minimum(rng.zipf(1.1, n), 30000) - 1
    k = rng.permutation(30000)[ranks].astype(np.int64)
    mask = rng.random(n) < 0.1
    if vkind == "int32_neg":
        v = pa.array(rng.integers(-3000, 2000, n).astype(np.int32), mask=mask)
    elif vkind == "int8":
        v = pa.array(rng.integers(-128, 128, n).astype(np.int8), mask=mask)
    elif vkind == "int16":
        v = pa.array(rng.integers(-30000, 30000, n).astype(np.int16))
    elif vkind == "uint8":
        v = pa.array(rng.integers(0, 256, n).astype(np.uint8), mask=mask)
    elif vkind == "uint32":
        v = pa.array(rng.integers(4_000_000_000, 4_000_100_000, n).astype(np.uint32))
    else:
        v = pa.array(rng.random(n) < 0.3, mask=mask)
    t = pa.table({"k": k, "v": v, "w": rng.normal(size=n)})
    aggs = [("v", "count_distinct", "nd"), ("v", "min", "mn"), ("v", "max", "mx"), ("v", "count", "c"),
            ("v", ("count_distinct", pc.CountOptions(mode="all")), "nda")]
    if other:
        aggs.append(("w", "sum", "ws"))
    res = run_groupby(t, ["k"], aggs)
    exp = R.groupby(t, ["k"], aggs)
    assert_tables_equal(res, exp, sort_by=["k"], rtol=RTOL)


# ---- partitioned plan (one fixed-width key, <= 2 fixed-width value columns) ----
PART_AGGS = [
    ("v", "sum", "s"), ("v", "mean", "m"), ("v", "count", "c"), (None, "count_all", "n"),
    ("v", "min", "vmin"), ("v", "max", "vmax"),
    ("v", ("count", pc.CountOptions(mode="all")), "c_all"),
    ("v", ("count", pc.CountOptions(mode="only_null")), "c_null"),
    ("i", "min", "mn"), ("i", "max", "mx"), ("i", "count_distinct", "nd"), ("i", "sum", "isum"),
    ("i", "mean", "imean"), ("i", ("count_distinct", pc.CountOptions(mode="all")), "nd_all"),
]


def _part_table(rng, n, key_kind, ngroups, zipf=None, key_null_p=0.01, i_null_p=0.05, ivals=1000):
    if zipf:
        raw = rng.permutation(ngroups)[np.minimum(rng.zipf(zipf, n), ngroups) - 1]
    else:
        raw = rng.integers(0, ngroups, n)
    k = pa.array(raw.astype(key_kind), mask=rng.random(n) < key_null_p if key_null_p else None)
    v = pa.array(rng.normal(size=n), mask=rng.random(n) < 0.1)
    i = pa.array(rng.integers(-ivals // 2, ivals, n).astype(np.int32), mask=rng.random(n) < i_null_p)
    return pa.table({"k": k, "v": v, "i": i})


@pytest.mark.parametrize("key_kind,ngroups,zipf,n", [
    ("int64", 50_000, 1.1, 600_000),     # hot keys in shared memory + cold buckets
    ("int32", 300_000, None, 500_000),   # mostly cold: many small buckets
    ("float64", 20_000, 1.3, 400_000),   # float keys by bit pattern
    ("int8", 200, None, 300_000),        # few groups: large buckets on global scratch
    ("uint64", 2_000, None, 2_000_000),  # large buckets, hot keys picked among equals
])
def test_groupby_partitioned_plan(monkeypatch, key_kind, ngroups, zipf, n):
    monkeypatch.setenv("LDF_B200_GB_PART", "1")
    monkeypatch.setenv("LDF_B200_GB_PART_MIN_ROWS", "0")
    rng = np.random.default_rng(ngroups + n)
    t = _part_table(rng, n, key_kind, ngroups, zipf=zipf)
    res = run_groupby(t, ["k"], PART_AGGS)
    exp = R.groupby(t, ["k"], PART_AGGS)
    assert_tables_equal(res, exp, sort_by=["k"], rtol=RTOL)


def test_groupby_partitioned_single_column_and_edge_keys(monkeypatch):
    monkeypatch.setenv("LDF_B200_GB_PART", "1")
    monkeypatch.setenv("LDF_B200_GB_PART_MIN_ROWS", "0")
    rng = np.random.default_rng(41)
    n = 400_000
    raw = rng.integers(0, 5000, n).astype(np.int64)
    raw[::97] = -1          # all-ones bits (the sample table's empty marker)
    raw[5::101] = 2**63 - 1
    t = pa.table({"k": raw, "x": pa.array(rng.integers(-2**40, 2**40, n), mask=rng.random(n) < 0.2)})
    aggs = [("x", "sum", "s"), ("x", "mean", "m"), ("x", "min", "mn"), ("x", "max", "mx"), (None, "count_all", "n")]
    assert_tables_equal(run_groupby(t, ["k"], aggs), R.groupby(t, ["k"], aggs), sort_by=["k"], rtol=RTOL)


def test_groupby_partitioned_falls_back_on_special_floats(monkeypatch):
    # NaN / inf / tiny values are outside the exact fixed-point range: the
    # call re-runs on the general plan, with the same results
    monkeypatch.setenv("LDF_B200_GB_PART", "1")
    monkeypatch.setenv("LDF_B200_GB_PART_MIN_ROWS", "0")
    rng = np.random.default_rng(43)
    t = _part_table(rng, 200_000, "int64", 3_000, zipf=1.2)
    v = t.column("v").to_numpy(zero_copy_only=False).copy()
    v[7], v[11], v[13] = np.nan, np.inf, 1e-300
    t = t.set_column(1, "v", pa.array(v, mask=np.isnan(v) & (np.arange(len(v)) != 7)))
    aggs = [("v", "sum", "s"), ("v", "mean", "m"), ("i", "count_distinct", "nd"), (None, "count_all", "n")]
    assert_tables_equal(run_groupby(t, ["k"], aggs), R.groupby(t, ["k"], aggs), sort_by=["k"], rtol=RTOL)
