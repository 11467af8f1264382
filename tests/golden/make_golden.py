"""Generate the golden fixtures of the relational hot path.

Two kinds of cases, all small:
  * known answers written out in the reference's own tests (explicit expected
    tables), transcribed with their file:line;
  * the reference's small/seeded test inputs with the expected output computed
    by the reference's CPU path (Arrow Acero / SortIndices through
    ``oracle.arrow_ref``, the same Arrow calls as the cpu_variant tasks).

Writes ``tests/golden/golden.arrows`` (one Arrow IPC stream per table, indexed
by ``tests/golden/manifest.json``).  Run from the repository root:
``python tests/golden/make_golden.py``.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import arrow_ref as A  # noqa: E402

OUT = Path(__file__).resolve().parent


def i32(v, mask=None):
    return pa.array(v, type=pa.int32(), mask=None if mask is None else ~np.asarray(mask, dtype=bool))


def s(v, valid=None):
    if valid is None:
        return pa.array(v, type=pa.string())
    return pa.array([x if ok else None for x, ok in zip(v, valid)], type=pa.string())


def cases():
    out = []

    # ---- join: cpp/tests/test_join.cpp ------------------------------------------
    def jc(name, src, lhs, rhs, lk, rk, how, nulls_equal=True, lo=None, ro=None, expected=None):
        if expected is None:
            expected = A.join(lhs, rhs, lk, rk, how, nulls_equal, lo, ro)
        out.append(dict(op="join", name=name, source=src, how=how, lhs_keys=lk, rhs_keys=rk,
                        nulls_equal=nulls_equal, lhs_out=lo, rhs_out=ro,
                        tables=dict(lhs=lhs, rhs=rhs, expected=expected)))

    t0 = pa.table({"a": i32([3, 1, 2, 0, 2]), "b": s(["s1", "s1", "s0", "s4", "s0"]), "c": i32([0, 1, 2, 4, 1])})
    t1 = pa.table({"d": i32([2, 2, 0, 4, 3]), "e": s(["s1", "s0", "s1", "s2", "s1"]), "f": i32([1, 0, 1, 2, 1])})
    jc("InnerJoinNoNulls", "cpp/tests/test_join.cpp:156-169", t0, t1, ["a", "b"], ["d", "e"], "inner")
    t0 = pa.table({"a": i32([3, 1, 2, 0, 3]), "b": s(["s0", "s1", "s2", "s4", "s1"]), "c": i32([0, 1, 2, 4, 1])})
    jc("InnerJoinOneMatch", "cpp/tests/test_join.cpp:171-184", t0, t1, ["a", "b"], ["d", "e"], "inner")
    t0 = pa.table({"a": i32([3, 1, 2, 0, 2]), "b": s(["s1", "s1", "s0", "s4", "s0"], [1, 1, 0, 1, 1]),
                   "c": i32([0, 1, 2, 4, 1])})
    t1n = pa.table({"d": i32([2, 2, 0, 4, 3]), "e": s(["s1", "s0", "s1", "s2", "s1"]),
                    "f": i32([1, 0, 1, 2, 1], mask=[1, 0, 1, 1, 1])})
    jc("InnerJoinWithNulls", "cpp/tests/test_join.cpp:186-202", t0, t1n, ["a", "b"], ["d", "e"], "inner")
    t0 = pa.table({"a": i32([1, 1, 0, 2, 0]), "b": s(["s1", "s1", "s0", "s2", "s0"], [1, 1, 0, 1, 1]),
                   "c": i32([0, 1, 2, 3, 4])})
    t1s = pa.table({"d": i32([1, 1, 2]), "e": s(["s1", "s1", "s2"]), "f": i32([1, 0, 1], mask=[1, 0, 1])})
    jc("InnerJoinDifferentLengths", "cpp/tests/test_join.cpp:204-220", t0, t1s, ["a", "b"], ["d", "e"], "inner")
    t0 = pa.table({"a": i32([3, 1, 2, 0, 3]), "b": s(["s0"] * 5), "c": i32([0, 1, 2, 4, 1])})
    t1c = pa.table({"d": i32([2, 2, 0, 4, 3]), "e": s(["s1"] * 5), "f": i32([1, 0, 1, 2, 1])})
    jc("LeftJoinNoNullsWithNoCommon", "cpp/tests/test_join.cpp:222-234", t0, t1c, ["a", "b"], ["d", "e"], "left")
    t0 = pa.table({"a": i32([3, 1, 2, 0, 3]), "b": s(["s0", "s1", "s2", "s4", "s1"]), "c": i32([0, 1, 2, 4, 1])})
    jc("LeftJoinNoNulls", "cpp/tests/test_join.cpp:236-248", t0, t1, ["a", "b"], ["d", "e"], "left")
    jc("FullJoinNoNulls", "cpp/tests/test_join.cpp:306-318", t0, t1, ["a", "b"], ["d", "e"], "full")
    t0 = pa.table({"a": i32([3, 1, 2, 0, 2]), "b": s(["s1", "s1", "", "s4", "s0"], [1, 1, 0, 1, 1]),
                   "c": i32([0, 1, 2, 4, 1])})
    for how in ("left", "anti", "semi"):
        jc(f"LeftAntiSemiJoinWithNulls_{how}", "cpp/tests/test_join.cpp:250-266", t0, t1n, ["a", "b"],
           ["d", "e"], how)
    # explicit expected table: LEFT join on null keys (test_join.cpp:269-304)
    l = pa.table({"a": i32([3, 1, 0], mask=[1, 0, 1]), "b": s(["s0", "s1", "s2"]), "c": i32([0, 1, 2])})
    r = pa.table({"d": i32([0, 5, 3, 7], mask=[1, 1, 1, 0]), "e": s(["s1", "s0", "s0", "s1"]),
                  "f": i32([1, 4, 2, 8])})
    exp = pa.table({"a": i32([1, 0, 3], mask=[0, 1, 1]), "b": s(["s1", "s2", "s0"]), "c": i32([1, 2, 0]),
                    "f": i32([8, 1, 2], mask=[1, 0, 1])})
    jc("LeftJoinOnNulls", "cpp/tests/test_join.cpp:269-304", l, r, ["a", "b"], ["d", "e"], "left", True,
       ["a", "b", "c"], ["f"], expected=exp)
    t0 = pa.table({"a": i32([3, 1, 2, 0, 3]), "b": s(["s0", "s1", "s2", "s4", "s1"]), "c": i32([0, 1, 2, 4, 1])})
    t1f = pa.table({"d": i32([2, 2, 0, 4, 3], mask=[1, 1, 1, 0, 1]), "e": s(["s1", "s0", "s1", "s2", "s1"]),
                    "f": i32([1, 0, 1, 2, 1])})
    jc("FullJoinWithNulls", "cpp/tests/test_join.cpp:320-334", t0, t1f, ["a", "b"], ["d", "e"], "full")
    # python/tests/test_join.py:156-178 (string keys, explicit expected)
    l = pa.table({"key": ["1", "2", "3"], "data0": [1, 2, 3]})
    r = pa.table({"key": ["3", "2", "1"], "data1": ["1", "2", "3"]})
    exp = pa.table({"data0": [1, 2, 3], "key": ["1", "2", "3"], "data1": ["3", "2", "1"]})
    jc("column_names_and_strings", "python/tests/test_join.py:156-178", l, r, ["key"], ["key"], "inner", True,
       ["data0", "key"], ["data1"], expected=exp)
    # python/tests/test_join.py:53-57 and :59-65 (duplicates, two-column keys)
    l = pa.table({"a": [1, 2, 3, 4, 5], "payload_a": np.arange(5)})
    r = pa.table({"b": [1, 1, 2, 2, 5, 6], "payload_b": np.arange(6) * -1})
    for how in ("inner", "left", "full", "semi", "anti"):
        for ne in (True, False):
            jc(f"dup_keys_{how}_{ne}", "python/tests/test_join.py:53-57", l, r, ["a"], ["b"], how, ne)
    l = pa.table({"a_a": [1, 2, 3, 4, 5], "b_a": [5, 4, 3, 2, 1]})
    r = pa.table({"a_b": [5, 4, 3, 2, 1], "b_b": [1, 2, 3, 4, 5]})
    jc("two_col_order", "python/tests/test_join.py:59-65", l, r, ["a_a", "b_a"], ["b_b", "a_b"], "inner")
    # python/tests/test_join.py:30-50 shape (shuffled aranges, payload nulls i%5==3), seeded here
    rng = np.random.default_rng(2024)
    for na, nb in ((60, 80), (80, 60)):
        a = rng.permutation(na).astype(np.int64)
        b = rng.permutation(nb).astype(np.int64)
        pay = pa.array(np.arange(na), mask=np.array([i % 5 == 3 for i in range(na)]))
        l = pa.table({"a": a, "payload_a": pay})
        r = pa.table({"b": b, "payload_b": np.arange(nb) * -1})
        ls = pa.table({"a": a, "payload_a": [str(i) for i in range(na)]})
        rs = pa.table({"b": b, "payload_b": [str(-i) for i in range(nb)]})
        for how in ("inner", "left", "full", "semi", "anti"):
            jc(f"arange_{na}_{nb}_{how}", "python/tests/test_join.py:30-50", l, r, ["a"], ["b"], how)
            jc(f"arange_str_{na}_{nb}_{how}", "python/tests/test_join.py:44-50", ls, rs, ["a"], ["b"], how)

    # ---- groupby: python/tests/test_groupby_aggregation.py --------------------------
    def gc(name, src, table, keys, aggs):
        exp = A.groupby(table, keys, aggs)
        aggs_j = []
        for in_col, kind, o in aggs:
            if isinstance(kind, tuple):
                kind = [kind[0], str(kind[1]).split("mode=")[-1].rstrip(")")]
            aggs_j.append([in_col, kind, o])
        out.append(dict(op="groupby", name=name, source=src, keys=keys, aggs=aggs_j,
                        tables=dict(table=table, expected=exp)))

    basic = [
        (["k1"], pa.table({"k1": ["x", "x", "y", "y", "z"], "d1": [1, 2, 0, 4, 1], "d2": [3, 2, 4, 5, 1]})),
        (["k1", "k2"], pa.table({"k1": ["x", "y", "y", "y", "x"], "d1": [1, 2, 0, 4, 1],
                                 "k2": ["y", "x", "y", "x", "y"], "d2": [3, 2, 4, 5, 1]})),
    ]
    for bi, (keys, tbl) in enumerate(basic):
        for ai, aggs in enumerate([[("d1", "sum", "sum")], [("d1", "min", "min"), ("d1", "max", "max")],
                                   [("d2", "mean", "mean")]]):
            gc(f"basic_{bi}_{ai}", "python/tests/test_groupby_aggregation.py:55-100", tbl, keys, aggs)
    for value_type in ("int64", "float64", "uint8"):
        for key_type in ("int64", "string", "float32"):
            for agg in ("sum", "min", "max", "count", "count_all", "mean", "count_distinct",
                        ("count_distinct", pc.CountOptions(mode="all"))):
                rng = np.random.RandomState(42)
                n_keys, n = 10, 1000
                if key_type == "int64":
                    key_a = pa.array(rng.randint(0, n_keys, n), type=pa.int64())
                elif key_type == "string":
                    key_a = pa.array([f"key_{i % n_keys}" for i in range(n)], type=pa.string())
                else:
                    key_a = pa.array(rng.randint(0, n_keys, n).astype(np.float32), type=pa.float32())
                key_b = pa.array(rng.randint(0, n_keys, n), type=pa.int64())
                value_a = pa.array(rng.random(n).astype(value_type), type=value_type)
                value_b = pa.array(rng.random(n), type=pa.float64())
                tbl = pa.Table.from_arrays([key_a, value_a, key_b, value_b],
                                           names=["key_a", "value_a", "key_b", "value_b"])
                an = agg if isinstance(agg, str) else agg[0] + "_all"
                aggs = [("value_a" if agg != "count_all" else None, agg, f"value_a_{an}"),
                        ("value_b" if agg != "count_all" else None, agg, f"value_b_{an}")]
                gc(f"numeric_{value_type}_{key_type}_{an}", "python/tests/test_groupby_aggregation.py:103-161",
                   tbl, ["key_a", "key_b"], aggs)

    # ---- sort: python/tests/test_sort.py ----------------------------------------
    def sc(name, src, table, keys, asc, nulls_at_end, limit=None, expected=None):
        if expected is None:
            expected = A.sort(table, keys, asc, nulls_at_end, limit)
        out.append(dict(op="sort", name=name, source=src, keys=keys, ascending=asc, nulls_at_end=nulls_at_end,
                        limit=limit, tables=dict(table=table, expected=expected)))

    exp = pa.table({"a": pa.array([None, None, 0, 1], type=pa.int64()),
                    "b": pa.array([None, 0, 1, None], type=pa.int64())})
    sc("na_position_explicit", "python/tests/test_sort.py:212-234",
       pa.table({"a": pa.array([0, 1, None, None], type=pa.int64()),
                 "b": pa.array([1, None, 0, None], type=pa.int64())}), ["a", "b"], [True, True], False, expected=exp)
    for by, asc, nl in ((["a"], [True], True), (["a"], [False], False), (["a", "b", "c"], [True, False, True], True),
                        (["c", "a", "b"], [True, False, True], False), (["c", "b", "a"], [True, False, True], True)):
        np.random.seed(1)
        repeats = 100
        va = np.arange(10).repeat(repeats)
        vb = np.arange(10.0).repeat(repeats)
        vc = ["a", "b", "hello", "d", "e", "f", "e", "\U0001F642", "e", "g"] * repeats
        np.random.shuffle(va)
        np.random.shuffle(vb)
        ma = np.random.choice([True, False], size=va.size, p=[0.1, 0.9])
        mb = np.random.choice([True, False], size=va.size, p=[0.1, 0.9])
        mc = np.random.choice([True, False], size=va.size, p=[0.1, 0.9])
        tbl = pa.table({"a": pa.array(va, mask=~ma), "b": pa.array(vb, mask=~mb), "c": pa.array(vc, mask=~mc),
                        "idx": np.arange(va.size)})
        sc("orders_" + "_".join(by) + f"_{nl}", "python/tests/test_sort.py:141-209", tbl, by, asc, nl)
    for i, values in enumerate([np.arange(0, 1000), np.arange(0, -1000, -1), np.ones(1000), np.ones(1)]):
        tbl = pa.table({"a": values, "b": np.arange(len(values))})
        sc(f"basic_{i}", "python/tests/test_sort.py:29-76", tbl, ["a"], [True], True)
    tbl = pa.table({"a": np.arange(0, 1000)})
    sc("limit_head", "python/tests/test_sort.py:79-89", tbl, ["a"], [True], True, 10)
    sc("limit_tail", "python/tests/test_sort.py:79-89", tbl, ["a"], [True], True, -10)
    for i in (0, 37, 149):
        values = np.concatenate([np.arange(i), np.full(50, i), np.arange(50 + i, 200)])
        for rev in (False, True):
            v = values[::-1].copy() if rev else values
            sc(f"shifted_window_{i}_{rev}", "python/tests/test_sort.py:113-140",
               pa.table({"a": v, "b": np.arange(200)}), ["a"], [True], True)
    return out


def main():
    manifest = []
    batches = []
    for c in cases():
        entry = {k: v for k, v in c.items() if k != "tables"}
        entry["tables"] = {}
        for tname, t in c["tables"].items():
            entry["tables"][tname] = len(batches)
            batches.append(t)
        manifest.append(entry)
    # one zstd-compressed IPC stream per table, concatenated; byte offsets in
    # the manifest give random access
    opts = pa.ipc.IpcWriteOptions(compression="zstd")
    offsets = []
    pos = 0
    with pa.OSFile(str(OUT / "golden.arrows"), "wb") as f:
        for t in batches:
            sink = pa.BufferOutputStream()
            with pa.ipc.new_stream(sink, t.schema, options=opts) as w:
                w.write_table(t)
            buf = sink.getvalue()
            f.write(buf)
            offsets.append([pos, buf.size])
            pos += buf.size
    (OUT / "manifest.json").write_text(json.dumps({"cases": manifest, "streams": offsets}, indent=1))
    print(f"{len(manifest)} cases, {len(batches)} tables, {pos} bytes")


if __name__ == "__main__":
    main()
