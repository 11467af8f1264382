"""distinct (stream_compaction.cpp:121-150): the distinct key combinations
equal the oracle's groups, and every output row is a whole input row (any
representative of its group), for int/float/string/multi-column keys with
nulls."""

import numpy as np
import pyarrow as pa
import pytest

from ldf_testing import assert_tables_equal, special_float_tables
from oracle import relational as R

pytestmark = pytest.mark.gpu


def run_distinct(t, keys):
    from legate_dataframe import LogicalTable
    from legate_dataframe.lib.stream_compaction import distinct

    return distinct(LogicalTable.from_arrow(t), keys).to_arrow()


def check(t, keys):
    res = run_distinct(t, keys)
    assert res.column_names == t.column_names
    exp_keys = R.groupby(t, keys, [])
    assert_tables_equal(res.select(keys), exp_keys, sort_by=keys)
    # every output row is an input row
    rows_in = set(zip(*[t.column(c).to_pylist() for c in t.column_names]))
    for row in zip(*[res.column(c).to_pylist() for c in res.column_names]):
        key = tuple(row)
        assert key in rows_in or any(isinstance(x, float) and x != x for x in key)


@pytest.mark.parametrize("kind", ["int64", "int32", "string", "float64"])
def test_distinct_single_key(kind):
    rng = np.random.default_rng(3)
    n = 20000
    raw = rng.integers(0, 500, n)
    mask = rng.random(n) < 0.05
    if kind == "string":
        k = pa.array([None if m else f"k{x}" for x, m in zip(raw, mask)])
    else:
        k = pa.array(raw.astype(kind), mask=mask)
    t = pa.table({"k": k, "v": rng.normal(size=n), "s": pa.array([f"s{i}" for i in range(n)]),
                  "i": pa.array(rng.integers(0, 9, n).astype(np.int16), mask=rng.random(n) < 0.1)})
    check(t, ["k"])


def test_distinct_multi_key_and_empty():
    rng = np.random.default_rng(4)
    n = 30000
    t = pa.table({"a": pa.array(rng.integers(0, 7, n).astype(np.int32), mask=rng.random(n) < 0.05),
                  "b": pa.array([f"x{v}" for v in rng.integers(0, 30, n)]),
                  "c": rng.integers(-5, 5, n)})
    check(t, ["a", "b"])
    check(t, ["c", "a"])
    e = pa.table({"a": pa.array([], pa.int64()), "b": pa.array([], pa.string())})
    assert run_distinct(e, ["a"]).num_rows == 0


def test_distinct_special_floats():
    t, _, _ = special_float_tables()
    res = run_distinct(t, ["k"])
    assert res.num_rows == 5  # 0.0, -0.0, NaN, -NaN, 1.0 (bit-pattern keys, as Arrow's grouper)


def test_distinct_known_answer():
    """The reference's hard-coded answer (cpp/tests/test_stream_compaction.cpp:50-74):
    distinct on ("a", "b"), then sorted by (a asc, b desc, c asc) with nulls
    first, through this library's own sort."""
    from legate_dataframe import LogicalTable
    from legate_dataframe.lib.sort import sort
    from legate_dataframe.lib.stream_compaction import distinct

    t = pa.table({"a": pa.array([0, 0, 0, 1, 1, 1], pa.int32(), mask=np.array([1, 1, 1, 0, 0, 0], bool)),
                  "b": pa.array(["this", "this", "string", "string", "col", "col"]),
                  "c": pa.array([0, 0, 2, 3, 4, 4], pa.float64())})
    res = distinct(LogicalTable.from_arrow(t), ["a", "b"])
    got = sort(res, ["a", "b", "c"], sort_ascending=[True, False, True], nulls_at_end=False).to_arrow()
    exp = pa.table({"a": pa.array([0, 0, 1, 1], pa.int32(), mask=np.array([1, 1, 0, 0], bool)),
                    "b": pa.array(["this", "string", "string", "col"]),
                    "c": pa.array([0, 2, 3, 4], pa.float64())})
    assert got.column_names == exp.column_names
    for name in exp.column_names:
        assert got.column(name).to_pylist() == exp.column(name).to_pylist(), name
    assert got.schema.field("a").type == pa.int32() and got.schema.field("c").type == pa.float64()
