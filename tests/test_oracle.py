"""Pin the CPU oracle: against the reference's golden vectors / known answers
and against the reference's own CPU path (Arrow Acero / SortIndices) on
seeded inputs.  CPU only."""

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

from ldf_testing import agg_spec, assert_tables_equal, load_golden, special_float_tables
from oracle import arrow_ref as A
from oracle import relational as R

CASES = list(load_golden())


@pytest.mark.parametrize("case", CASES, ids=[c["op"] + ":" + c["name"] for c in CASES])
def test_oracle_matches_golden(case):
    t = case["tables"]
    if case["op"] == "join":
        res = R.join(t["lhs"], t["rhs"], case["lhs_keys"], case["rhs_keys"], case["how"], case["nulls_equal"],
                     case["lhs_out"], case["rhs_out"])
        assert_tables_equal(res, t["expected"], check_types=False)
    elif case["op"] == "groupby":
        res = R.groupby(t["table"], case["keys"], agg_spec(case["aggs"]))
        assert_tables_equal(res, t["expected"], sort_by=case["keys"], rtol=1e-12)
    else:
        res = R.sort(t["table"], case["keys"], case["ascending"], case["nulls_at_end"], case["limit"])
        assert_tables_equal(res, t["expected"], sort_by=None)


def _random_table(rng, n, key_type, null_p, nkeys=1, prefix="k", key_range=50):
    cols = {}
    for j in range(nkeys):
        mask = rng.random(n) < null_p if null_p else None
        if key_type == "string":
            vals = [f"s{v}" for v in rng.integers(0, key_range, n)]
            cols[f"{prefix}{j}"] = pa.array([None if (mask is not None and m) else v for v, m in
                                            zip(vals, mask if mask is not None else [False] * n)], pa.string())
        else:
            vals = rng.integers(0, key_range, n).astype(key_type)
            cols[f"{prefix}{j}"] = pa.array(vals, mask=mask)
    cols[prefix + "_pay"] = pa.array(rng.normal(size=n), mask=rng.random(n) < 0.1)
    cols[prefix + "_ipay"] = pa.array(rng.integers(-1000, 1000, n).astype(np.int32))
    return pa.table(cols)


@pytest.mark.parametrize("how", ["inner", "left", "full", "semi", "anti"])
@pytest.mark.parametrize("nulls_equal", [True, False])
@pytest.mark.parametrize("key_type", ["int32", "int64", "string"])
@pytest.mark.parametrize("nkeys", [1, 2])
def test_oracle_join_vs_arrow(how, nulls_equal, key_type, nkeys):
    rng = np.random.default_rng(11 + nkeys)
    lhs = _random_table(rng, 300, key_type, 0.1, nkeys, "l", 40)
    rhs = _random_table(rng, 200, key_type, 0.1, nkeys, "r", 40)
    lk = [f"l{j}" for j in range(nkeys)]
    rk = [f"r{j}" for j in range(nkeys)]
    exp = A.join(lhs, rhs, lk, rk, how, nulls_equal)
    res = R.join(lhs, rhs, lk, rk, how, nulls_equal)
    assert_tables_equal(res, exp, check_types=False)


@pytest.mark.parametrize("key_type", ["int64", "string", "float32"])
def test_oracle_groupby_vs_arrow(key_type):
    rng = np.random.default_rng(5)
    n = 2000
    t = _random_table(rng, n, key_type if key_type != "float32" else "int64", 0.05, 2, "k", 12)
    if key_type == "float32":
        t = t.set_column(0, "k0", pc.cast(t.column("k0"), pa.float32()))
    aggs = [("k_pay", "sum", "s"), ("k_pay", "mean", "m"), ("k_pay", "count", "c"), (None, "count_all", "ca"),
            ("k_ipay", "min", "mn"), ("k_ipay", "max", "mx"), ("k_ipay", "count_distinct", "nd"),
            ("k_pay", ("count", pc.CountOptions(mode="all")), "call"),
            ("k_pay", ("count", pc.CountOptions(mode="only_null")), "cnull"),
            ("k_ipay", ("count_distinct", pc.CountOptions(mode="all")), "ndall"), ("k_ipay", "sum", "isum")]
    exp = A.groupby(t, ["k0", "k1"], aggs)
    res = R.groupby(t, ["k0", "k1"], aggs)
    assert_tables_equal(res, exp, sort_by=["k0", "k1"], rtol=1e-12)


@pytest.mark.parametrize("nulls_at_end", [True, False])
@pytest.mark.parametrize("asc", [[True, True, True], [False, True, False], [True, False, True]])
def test_oracle_sort_vs_arrow(nulls_at_end, asc):
    rng = np.random.default_rng(3)
    n = 3000
    t = pa.table({
        "a": pa.array(rng.integers(0, 20, n), mask=rng.random(n) < 0.1),
        "b": pa.array(rng.integers(0, 5, n).astype(np.float64), mask=rng.random(n) < 0.1),
        "c": pa.array([None if m else f"x{v}" for v, m in zip(rng.integers(0, 30, n), rng.random(n) < 0.1)]),
        "idx": np.arange(n),
    })
    keys = ["c", "a", "b"]
    exp = A.sort(t, keys, asc, nulls_at_end)
    res = R.sort(t, keys, asc, nulls_at_end)
    assert_tables_equal(res, exp, sort_by=None)


def test_oracle_partition_properties():
    rng = np.random.default_rng(9)
    n = 5000
    t = pa.table({"k": pa.array(rng.integers(0, 300, n), mask=rng.random(n) < 0.05),
                  "s": [f"v{v}" for v in rng.integers(0, 100, n)], "i": np.arange(n)})
    out, offsets, bucket = R.hash_partition(t, ["k", "s"], 16)
    assert offsets[0] == 0 and offsets[-1] == n
    # permutation of the input, stable within buckets, equal keys in one bucket
    idx = np.asarray(out.column("i"))
    assert sorted(idx.tolist()) == list(range(n))
    for b in range(16):
        seg = idx[offsets[b]:offsets[b + 1]]
        assert np.all(np.diff(seg) > 0)
        assert np.all(bucket[seg] == b)
    keys = list(zip(t.column("k").to_pylist(), t.column("s").to_pylist()))
    seen = {}
    for i, kk in enumerate(keys):
        assert seen.setdefault(kk, bucket[i]) == bucket[i]


def test_oracle_hash_known_answers():
    # MurmurHash3 fmix64 of small integers (independent big-int restatement)
    def fmix(x):
        m = (1 << 64) - 1
        x ^= x >> 33
        x = (x * 0xFF51AFD7ED558CCD) & m
        x ^= x >> 33
        x = (x * 0xC4CEB9FE1A85EC53) & m
        x ^= x >> 33
        return x

    xs = np.array([0, 1, 2, 12345, (1 << 64) - 1], dtype=np.uint64)
    got = R._mix64(xs)
    assert [int(g) for g in got] == [fmix(int(x)) for x in xs]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_special_float_keys_vs_arrow(dtype):
    t, lhs, rhs = special_float_tables(dtype)
    aggs = [("v", "sum", "s"), ("w", "count_distinct", "nd")]
    a = R.groupby(t, ["k"], aggs)
    b = A.groupby(t, ["k"], aggs)
    assert a.num_rows == b.num_rows == 5  # 0.0, -0.0, NaN, -NaN, 1.0
    assert_tables_equal(a, b, sort_by=["s"])
    for how in ("inner", "left", "full", "semi", "anti"):
        exp = A.join(lhs, rhs, ["k"], ["k2"], how, True)
        res = R.join(lhs, rhs, ["k"], ["k2"], how, True)
        assert_tables_equal(res, exp, sort_by=[c for c in exp.column_names if c in ("a", "b")], check_types=False)


def test_oracle_string_hashes_vectorized():
    # the vectorized string hash (used at full size) equals the byte-wise
    # definition on strings of every length class, tails included
    rng = np.random.default_rng(11)
    strs = [bytes(rng.integers(48, 123, int(n))) for n in rng.integers(0, 41, 2000)] + [b"", b"x" * 8, b"y" * 24]
    off = np.zeros(len(strs) + 1, np.int64)
    off[1:] = np.cumsum([len(s) for s in strs])
    got = R.string_hashes(np.frombuffer(b"".join(strs), np.uint8), off)
    assert [int(g) for g in got] == [R._hash_bytes(s) for s in strs]


def test_oracle_segment_sums_c():
    # the C Neumaier segment sums agree with math.fsum (exactly rounded)
    import math

    from oracle import native

    rng = np.random.default_rng(12)
    x = rng.normal(size=30000) * np.exp(rng.normal(size=30000) * 8)
    x = np.concatenate([x, -x[:20000] * (1 + 1e-15)])
    valid = (rng.random(len(x)) >= 0.1).astype(np.uint8)
    off = np.concatenate([[0], np.sort(rng.choice(np.arange(1, len(x)), 40, replace=False)), [len(x)]])
    sums, cnt = native.segment_sums(x, valid, off)
    for s in range(len(off) - 1):
        seg = x[off[s]:off[s + 1]][valid[off[s]:off[s + 1]] == 1]
        exact = math.fsum(seg)
        assert cnt[s] == len(seg)
        assert abs(sums[s] - exact) <= 1e-12 * abs(exact) + 1e-300
    s32, c32 = native.segment_sums(x.astype(np.float32), None, off)
    assert abs(s32[0] - math.fsum(x[:off[1]].astype(np.float32).astype(np.float64))) <= 1e-12 * abs(s32[0])


def test_oracle_float_sums_with_infinities_vs_arrow():
    # +inf / -inf / NaN values propagate as in Arrow's hash_sum
    k = np.array([0, 0, 1, 1, 2, 2, 3, 3, 4], dtype=np.int64)
    v = np.array([np.inf, 1.0, -np.inf, 2.0, np.inf, -np.inf, np.nan, 1.0, 5.0])
    t = pa.table({"k": k, "v": v})
    aggs = [("v", "sum", "s"), ("v", "mean", "m")]
    assert_tables_equal(R.groupby(t, ["k"], aggs), A.groupby(t, ["k"], aggs), sort_by=["k"])


def test_oracle_distinct_known_answer():
    """The oracle's distinct keys (its groupby with no aggregation) against the
    reference's hard-coded answer (cpp/tests/test_stream_compaction.cpp:50-74)."""
    t = pa.table({"a": pa.array([0, 0, 0, 1, 1, 1], pa.int32(), mask=np.array([1, 1, 1, 0, 0, 0], bool)),
                  "b": pa.array(["this", "this", "string", "string", "col", "col"])})
    got = R.sort(R.groupby(t, ["a", "b"], []), ["a", "b"], ascending=[True, False], nulls_at_end=False)
    assert got.column("a").to_pylist() == [None, None, 1, 1]
    assert got.column("b").to_pylist() == ["this", "string", "string", "col"]
