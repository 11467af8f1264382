"""Arrow / Parquet / CSV data into the device layout: Arrow buffers are
copied as they are and the validity bitmaps and string offsets are expanded
on the device (ldf_b200_arrow_bits_to_bytes, ldf_b200_arrow_offsets_to_ranges).
Round trips must give back the Arrow input exactly, including sliced arrays
(non-zero offsets, bitmaps that start mid-byte) and int64 string offsets."""

import numpy as np
import pyarrow as pa
import pyarrow.csv as pacsv
import pyarrow.parquet as pq
import pytest

from ldf_testing import assert_tables_equal
from oracle import relational as R

pytestmark = pytest.mark.gpu


def _table(n, seed=0):
    rng = np.random.default_rng(seed)
    mask = rng.random(n) < 0.2
    return pa.table({
        "i8": pa.array(rng.integers(-100, 100, n).astype(np.int8), mask=mask),
        "i32": pa.array(rng.integers(-1000, 1000, n).astype(np.int32)),
        "i64": pa.array(rng.integers(-(2**40), 2**40, n), mask=rng.random(n) < 0.5),
        "u16": pa.array(rng.integers(0, 60000, n).astype(np.uint16)),
        "f32": pa.array(rng.normal(size=n).astype(np.float32), mask=mask),
        "f64": pa.array(rng.normal(size=n)),
        "b": pa.array(rng.random(n) < 0.5, mask=rng.random(n) < 0.1),
        "b2": pa.array(rng.random(n) < 0.5),
        "s": pa.array([None if m else "x" * (i % 13) + str(i) for i, m in enumerate(rng.random(n) < 0.15)],
                      type=pa.string()),
        "ls": pa.array(["é" * (i % 5) + str(i) for i in range(n)], type=pa.large_string()),
        "ts": pa.array(rng.integers(0, 2**50, n), type=pa.timestamp("us"), mask=rng.random(n) < 0.05),
        "d": pa.array(rng.integers(0, 20000, n).astype(np.int32), type=pa.date32()),
    })


@pytest.mark.parametrize("n", [0, 1, 7, 8, 9, 1000, 100_003])
def test_from_arrow_roundtrip(n):
    from legate_dataframe import LogicalTable

    t = _table(n, seed=n)
    assert LogicalTable.from_arrow(t).to_arrow().equals(t)


@pytest.mark.parametrize("start,length", [(1, 50), (3, 1000), (8, 997), (13, 1), (100, 0), (5, 2000)])
def test_from_arrow_sliced(start, length):
    """Offsets that are not multiples of 8 make the bitmaps start mid-byte."""
    from legate_dataframe import LogicalTable

    t = _table(3000, seed=start).slice(start, length)
    assert LogicalTable.from_arrow(t).to_arrow().equals(t)


def test_from_arrow_chunked():
    from legate_dataframe import LogicalTable

    a, b = _table(500, 1), _table(700, 2)
    t = pa.concat_tables([a, b])
    assert t.column("s").num_chunks == 2
    assert LogicalTable.from_arrow(t).to_arrow().equals(t.combine_chunks())


def test_parquet_read_write(tmp_path):
    from legate_dataframe.lib.groupby_aggregation import groupby_aggregation
    from legate_dataframe.lib.parquet import parquet_read, parquet_write

    parts = [_table(4000, seed=s) for s in range(3)]
    for i, p in enumerate(parts):
        pq.write_table(p, tmp_path / f"in.{i}.parquet", row_group_size=1000)
    t = pa.concat_tables(parts)
    got = parquet_read(str(tmp_path / "in.*.parquet"))
    assert got.to_arrow().equals(t.combine_chunks())
    sub = parquet_read([tmp_path / "in.0.parquet"], columns=["s", "i64"])
    assert sub.to_arrow().equals(parts[0].select(["s", "i64"]))
    # an op on the ingested layout
    aggs = [("i64", "sum", "sum"), ("f64", "mean", "mean"), ("i32", "count_distinct", "nd")]
    res = groupby_aggregation(got, ["s"], aggs).to_arrow()
    assert_tables_equal(res, R.groupby(t.combine_chunks(), ["s"], aggs), sort_by=["s"], rtol=1e-12)
    parquet_write(got, tmp_path / "out")
    assert pq.read_table(tmp_path / "out" / "part.0.parquet").equals(t.combine_chunks())


def test_csv_read_write(tmp_path):
    from legate_dataframe.lib.csv import csv_read, csv_write

    rng = np.random.default_rng(4)
    n = 5000
    t = pa.table({"a": pa.array(rng.integers(-50, 50, n), mask=rng.random(n) < 0.1),
                  "b": pa.array(rng.normal(size=n)),
                  "c": pa.array([f"w{i % 97}" for i in range(n)])})
    pacsv.write_csv(t, tmp_path / "x.csv")
    got = csv_read(tmp_path / "x.csv", dtypes=[pa.int64(), pa.float64(), pa.string()], usecols=["a", "b", "c"])
    assert got.to_arrow().equals(t)
    two = csv_read(str(tmp_path / "x.csv"), dtypes="int64", names=["a"])
    assert two.to_arrow().equals(t.select(["a"]))
    # no header: integral usecols and names
    pacsv.write_csv(t, tmp_path / "nh.csv", write_options=pacsv.WriteOptions(include_header=False))
    got = csv_read(tmp_path / "nh.csv", dtypes=[pa.string(), pa.int64()], usecols=[2, 0], names=["c", "a"])
    assert got.to_arrow().equals(t.select(["c", "a"]))
    csv_write(got, tmp_path / "out", delimiter="|")
    back = pacsv.read_csv(tmp_path / "out" / "part.0.csv", parse_options=pacsv.ParseOptions(delimiter="|"))
    assert back.column("a").equals(t.column("a"))
