"""Parity of the sm_100a onesweep radix sort (through the C ABI) with the
oracle and golden vectors: multi-key, per-key direction, nulls first/last,
NaN, strings (bytewise, shorter prefix first), limits, stability."""

import numpy as np
import pyarrow as pa
import pytest

from ldf_testing import assert_tables_equal, load_golden
from oracle import relational as R

pytestmark = pytest.mark.gpu

SORT_CASES = [c for c in load_golden() if c["op"] == "sort"]


def run_sort(table, keys, asc=None, nulls_at_end=True, stable=True, limit=None):
    from legate_dataframe import LogicalTable
    from legate_dataframe.lib.sort import sort

    return sort(LogicalTable.from_arrow(table), keys, sort_ascending=asc, nulls_at_end=nulls_at_end,
                stable=stable, limit=limit).to_arrow()


@pytest.mark.parametrize("case", SORT_CASES, ids=[c["name"] for c in SORT_CASES])
def test_sort_golden(case):
    t = case["tables"]
    res = run_sort(t["table"], case["keys"], case["ascending"], case["nulls_at_end"], True, case["limit"])
    assert_tables_equal(res, t["expected"], sort_by=None)


@pytest.mark.parametrize("dtype", ["int8", "int16", "int32", "int64", "uint32", "uint64", "float32", "float64"])
@pytest.mark.parametrize("asc", [True, False])
@pytest.mark.parametrize("nulls_at_end", [True, False])
def test_sort_single_key_types(dtype, asc, nulls_at_end):
    rng = np.random.default_rng(42)
    n = 50_000
    if dtype.startswith("float"):
        v = (rng.normal(size=n) * 1e3).astype(dtype)
        v[::97] = np.nan
        v[::101] = -0.0
        v[::103] = np.inf
        v[::107] = -np.inf
    else:
        info = np.iinfo(dtype)
        v = rng.integers(info.min, info.max, n, dtype=dtype, endpoint=True)
        v[::50] = info.max
        v[::51] = info.min
    t = pa.table({"a": pa.array(v, mask=rng.random(n) < 0.05), "row": np.arange(n)})
    res = run_sort(t, ["a"], [asc], nulls_at_end)
    exp = R.sort(t, ["a"], [asc], nulls_at_end)
    # -0.0 == 0.0 ties keep input order; compare the row column exactly
    assert res.column("row").equals(exp.column("row"))


@pytest.mark.parametrize("asc", [[True, False], [False, True], [True, True]])
def test_sort_string_and_timestamp(asc):
    rng = np.random.default_rng(8)
    n = 100_000
    words = [("".join(rng.choice(list("abcdefghij0"), size=rng.integers(0, 20)))) for _ in range(3000)]
    words += ["ab", "ab\x00", "abc", "", "\U0001F642", "zz" * 20]
    s = pa.array([None if m else words[i] for i, m in zip(rng.integers(0, len(words), n), rng.random(n) < 0.03)])
    ts = pa.array(rng.integers(1_700_000_000_000_000, 1_700_000_000_000_000 + 31_536_000_000_000, n),
                  type=pa.timestamp("us"))
    t = pa.table({"s": s, "ts": ts, "v": rng.random(n).astype(np.float32), "row": np.arange(n)})
    for nulls_at_end in (True, False):
        res = run_sort(t, ["s", "ts"], asc, nulls_at_end)
        exp = R.sort(t, ["s", "ts"], asc, nulls_at_end)
        assert_tables_equal(res, exp, sort_by=None)


@pytest.mark.parametrize("case", ["fits64", "fits72", "too_wide", "limit", "string_ts"])
def test_sort_fused_key_word(case):
    """Keys without nulls or floats whose value ranges fit 72 bits are sorted
    on one fused word (every key loaded in input order by the first pass,
    carried through the others): mixed directions, negative values, ties on
    every key, a word over 64 bits (its low byte sorted on its own), one over
    72 bits (per-key passes), a limit, and a string key with a timestamp."""
    rng = np.random.default_rng(31)
    n = 1_000_003
    a = rng.integers(-50, 51, n).astype(np.int8)
    b = rng.integers(0, 1_000, n).astype(np.int32)
    if case == "fits64":
        c = rng.integers(-(2**30), 2**30, n)
    elif case == "too_wide":
        c = rng.integers(-(2**62), 2**62, n)
    else:
        c = 1_700_000_000_000_000 + rng.integers(0, 2**50, n)
    t = pa.table({"a": a, "b": b, "c": c, "row": np.arange(n)})
    if case == "string_ts":
        words = np.array([f"w{i * 7919 % 10007:05d}{'x' * (i % 5)}" for i in range(20_000)], dtype=object)
        t = pa.table({"s": pa.array(words[rng.integers(0, 20_000, n)]),
                      "ts": pa.array(c, type=pa.timestamp("us")), "row": np.arange(n)})
        res = run_sort(t, ["s", "ts"], [True, False])
        assert_tables_equal(res, R.sort(t, ["s", "ts"], [True, False]), sort_by=None)
        return
    limit = 1000 if case == "limit" else None
    res = run_sort(t, ["a", "b", "c"], [False, True, False], limit=limit)
    assert_tables_equal(res, R.sort(t, ["a", "b", "c"], [False, True, False], limit=limit), sort_by=None)


def test_sort_stability_many_ties():
    rng = np.random.default_rng(2)
    n = 300_000
    t = pa.table({"a": rng.integers(0, 3, n), "b": pa.array(rng.integers(0, 2, n), mask=rng.random(n) < 0.3),
                  "row": np.arange(n)})
    res = run_sort(t, ["a", "b"], [False, True], True, stable=False)
    exp = R.sort(t, ["a", "b"], [False, True], True)
    assert_tables_equal(res, exp, sort_by=None)


def test_sort_limits_and_empty():
    t = pa.table({"a": np.arange(1000)[::-1].copy(), "s": [str(i) for i in range(1000)]})
    for lim in (10, -10, 0, 999, 1000, 5000, -5000):
        res = run_sort(t, ["a"], limit=lim)
        exp = R.sort(t, ["a"], limit=lim)
        assert_tables_equal(res, exp, sort_by=None)
    e = pa.table({"a": pa.array([], pa.int64())})
    assert run_sort(e, ["a"]).num_rows == 0
    one = pa.table({"a": [5]})
    assert run_sort(one, ["a"]).to_pydict() == {"a": [5]}


def test_sort_all_equal_skips_passes():
    t = pa.table({"a": np.full(10000, 7, dtype=np.int64), "row": np.arange(10000)})
    res = run_sort(t, ["a"])
    assert res.column("row").to_pylist() == list(range(10000))


@pytest.mark.parametrize("n", [3_000_000, 3072 * 1000])
def test_sort_many_tiles_per_block(n):
    """Thousands of onesweep tiles per pass (long look-back chains, the
    look-back loading several predecessors per round trip), with and without a
    partial last tile; two keys so the second key's first pass gathers
    through the permutation."""
    rng = np.random.default_rng(11)
    t = pa.table({"k": rng.integers(-(2**63), 2**63 - 1, n, dtype=np.int64),
                  "u": pa.array(rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)),
                  "row": np.arange(n)})
    res = run_sort(t, ["k"])
    assert_tables_equal(res, R.sort(t, ["k"]), sort_by=None)
    res = run_sort(t, ["u", "k"], [False, True])
    assert_tables_equal(res, R.sort(t, ["u", "k"], [False, True]), sort_by=None)


def test_sort_strings_sampled_dictionary():
    """More than 4M string rows: the dedupe table of distinct strings is
    sized from a sampled estimate.  Checked by properties at this size:
    the keys come out in bytewise order, equal keys keep their input order,
    and the rows are a permutation of the input."""
    rng = np.random.default_rng(12)
    n, nd = 5_000_000, 300_000
    words = np.array([f"{i:x}{'z' * (i % 11)}" for i in range(nd)], dtype=object)
    ranks = np.minimum(rng.zipf(1.05, n), nd) - 1
    t = pa.table({"k": pa.array(words[ranks], pa.string()), "row": np.arange(n)})
    res = run_sort(t, ["k"])
    keys = np.array(res.column("k").to_pylist(), dtype=object)
    rows = res.column("row").to_numpy()
    assert np.array_equal(np.sort(rows), np.arange(n))
    assert np.array_equal(keys, words[ranks][rows])
    enc = np.array([k.encode() for k in keys], dtype=object)
    assert all(enc[i] <= enc[i + 1] for i in range(n - 1))
    same = enc[1:] == enc[:-1]
    assert np.all(rows[1:][same] > rows[:-1][same])


def test_sort_strings_dictionary_overflow_redo():
    """20M distinct strings: every string of the sample is seen once, so the
    sampled estimate (about 4.6M) is too low, the first dedupe table
    overflows (inserts stop early) and the ranking is redone with room for
    every row."""
    n = 20_000_000
    perm = np.random.default_rng(13).permutation(n)
    digits = np.stack([(perm // 10 ** (7 - d)) % 10 + 48 for d in range(8)], axis=1).astype(np.uint8)
    offsets = np.arange(0, 8 * n + 1, 8, dtype=np.int32)
    keys = pa.StringArray.from_buffers(n, pa.py_buffer(offsets), pa.py_buffer(digits.tobytes()))
    t = pa.table({"k": keys, "row": np.arange(n)})
    res = run_sort(t, ["k"])
    assert np.array_equal(res.column("row").to_numpy(), np.argsort(perm))
    out = res.column("k").combine_chunks()
    assert out.slice(0, 3).to_pylist() == ["00000000", "00000001", "00000002"]
    assert out[n - 1].as_py() == f"{n - 1:08d}"


def test_sort_wide_table_moved_and_gathered_columns():
    """A whole-table sort moves the first four columns inside its last radix
    pass (fixed widths straight into the outputs, a string column's ranges
    through scratch) and gathers the others through the permutation: every
    fixed width with and without nulls, strings on both sides of that
    boundary, and a constant key (no pass runs, the columns are copied)."""
    rng = np.random.default_rng(21)
    n = 200_000
    words = np.array([f"w{i:x}" + "q" * (i % 23) for i in range(5000)], dtype=object)

    def strings(null_frac):
        w = words[rng.integers(0, len(words), n)]
        return pa.array(w, pa.string(), mask=rng.random(n) < null_frac if null_frac else None)

    t = pa.table({
        "s1": strings(0.05),
        "i8": pa.array(rng.integers(-128, 128, n).astype(np.int8), mask=rng.random(n) < 0.1),
        "f32": rng.normal(size=n).astype(np.float32),
        "i16": pa.array(rng.integers(-300, 300, n).astype(np.int16), mask=rng.random(n) < 0.02),
        "s2": strings(0.0),
        "i64": pa.array(rng.integers(-(2**40), 2**40, n), mask=rng.random(n) < 0.03),
        "s3": strings(0.2),
        "row": np.arange(n),
    })
    for keys, asc in ((["i16", "s1"], [True, False]), (["i64"], [False]), (["s2", "f32"], [True, True])):
        for nulls_at_end in (True, False):
            res = run_sort(t, keys, asc, nulls_at_end)
            assert_tables_equal(res, R.sort(t, keys, asc, nulls_at_end), sort_by=None)
    const = t.append_column("c", pa.array(np.zeros(n, np.int32)))
    assert_tables_equal(run_sort(const, ["c"]), const, sort_by=None)


@pytest.mark.parametrize("const_key", [False, True])
def test_sort_packed_payload_records(const_key):
    """Non-nullable fixed-width columns among the four the last pass moves
    (a string key's representative rows included) travel packed in one
    16-byte record per row: 8+4+4 bytes with a string key, 8+4+2+1 bytes of
    integers; a constant key runs no pass and copies the records in order."""
    rng = np.random.default_rng(31)
    n = 150_000
    words = np.array([f"k{i}" + "x" * (i % 17) for i in range(3000)], dtype=object)
    key = np.zeros(n, np.int32) if const_key else rng.integers(0, 50, n).astype(np.int32)
    t1 = pa.table({
        "s": pa.array(words[rng.integers(0, len(words), n)], pa.string(), mask=rng.random(n) < 0.04),
        "ts": rng.integers(-(2**62), 2**62, n),
        "v": rng.normal(size=n).astype(np.float32),
        "h": rng.integers(-(2**15), 2**15, n).astype(np.int16),
        "k": key,
        "row": np.arange(n),
    })
    t2 = pa.table({
        "b": rng.integers(-128, 128, n).astype(np.int8),
        "h": rng.integers(-(2**15), 2**15, n).astype(np.int16),
        "i": rng.integers(-(2**31), 2**31, n).astype(np.int32),
        "l": rng.integers(-(2**63), 2**63 - 1, n, dtype=np.int64),
        "k": key,
        "row": np.arange(n),
    })
    for t, keys in ((t1, ["k", "s"] if not const_key else ["k"]), (t1, ["s"]), (t2, ["k", "h"]), (t2, ["k"])):
        for asc in (True, False):
            res = run_sort(t, keys, [asc] * len(keys))
            assert_tables_equal(res, R.sort(t, keys, [asc] * len(keys), True), sort_by=None)
