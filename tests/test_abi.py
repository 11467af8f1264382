"""The C-ABI library: loads, exports every symbol include/ldf_b200.h declares,
rejects bad arguments with status codes, and the Python mirror validates its
arguments like the reference.  CPU only: no kernel is launched here."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pyarrow as pa
import pytest
import torch

from legate_dataframe import LogicalTable
from legate_dataframe import _native as N
from legate_dataframe.lib.groupby_aggregation import groupby_aggregation
from legate_dataframe.lib.join import BroadcastInput, JoinType, join
from legate_dataframe.lib.sort import sort

HEADER = Path(__file__).resolve().parents[1] / "include" / "ldf_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(ldf_b200_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = N.lib()
    names = declared_functions()
    assert len(names) >= 7
    for name in names:
        assert hasattr(L, name), name
    assert b"sm_100a" in L.ldf_b200_version()


def test_struct_layout_matches_header():
    assert ctypes.sizeof(N.ldf_column) == 56
    assert ctypes.sizeof(N.ldf_aggregation) == 16
    assert ctypes.sizeof(N.ldf_allocator) == 24


def test_invalid_arguments_return_status_without_gpu():
    L = N.lib()
    out = (N.ldf_column * 1)()
    st = L.ldf_b200_join(None, -1, None, 0, None, None, 0, 0, 1, None, 0, None, 0, out, None, None)
    assert st == N.LDF_ERR_INVALID_ARGUMENT
    assert b"negative column count" in L.ldf_b200_last_error()
    cols = (N.ldf_column * 2)()
    cols[0].type, cols[0].size, cols[0].data = N.LDF_INT64, 4, 1
    cols[1].type, cols[1].size, cols[1].data = N.LDF_INT64, 5, 1
    st = L.ldf_b200_sort(cols, 2, N.int32_array([0]), (ctypes.c_uint8 * 1)(1), 1, 1, 0, -(2**63), out, None, None)
    assert st == N.LDF_ERR_INVALID_ARGUMENT
    assert b"differ in length" in L.ldf_b200_last_error()
    cols[1].size = 4
    cols[1].type = 99
    st = L.ldf_b200_hash_partition(cols, 2, N.int32_array([0]), 1, 4, out, (ctypes.c_int64 * 5)(), None, None)
    assert st == N.LDF_ERR_UNSUPPORTED
    with pytest.raises(ValueError):
        N.check(st)


def _cpu_table(t: pa.Table) -> LogicalTable:
    return LogicalTable.from_arrow(t, device=torch.device("cpu"))


def test_python_sort_argument_errors():
    # python/tests/test_sort.py:237-252
    tbl = _cpu_table(pa.table({"a": [0, 1, 2, 3], "b": [0, 1, 2, 3]}))
    for keys, asc in (([], None), (["bad_col"], None), (["a"], [True, False]), (["a", "b"], [True]),
                      (["a", "a"], [True, True])):
        with pytest.raises((ValueError, TypeError)):
            sort(tbl, keys=keys, sort_ascending=asc)


def test_python_join_argument_errors():
    l = _cpu_table(pa.table({"a": [1, 2], "x": [1, 2]}))
    r = _cpu_table(pa.table({"b": [1, 2], "y": [3, 4]}))
    with pytest.raises(ValueError):
        join(l, r, lhs_keys=["a"], rhs_keys=["b", "y"], join_type=JoinType.INNER)
    with pytest.raises(ValueError):  # duplicate output names
        join(l, r, lhs_keys=["a"], rhs_keys=["b"], join_type=JoinType.INNER, lhs_out_columns=["a"],
             rhs_out_columns=["b", "b"])
    with pytest.raises(ValueError):
        join(l, r, lhs_keys=["a"], rhs_keys=["b"], join_type=JoinType.SEMI, rhs_out_columns=["y"])
    # broadcast legality (join.cpp:386-396, python/tests/test_join.py:101-118)
    for how, bc in ((JoinType.FULL, BroadcastInput.LEFT), (JoinType.FULL, BroadcastInput.RIGHT),
                    (JoinType.LEFT, BroadcastInput.LEFT), (JoinType.SEMI, BroadcastInput.LEFT),
                    (JoinType.ANTI, BroadcastInput.LEFT)):
        with pytest.raises(RuntimeError):
            join(l, r, lhs_keys=["a"], rhs_keys=["b"], join_type=how, broadcast=bc)


def test_python_groupby_argument_errors():
    t = _cpu_table(pa.table({"k": [1, 2], "v": [1.0, 2.0]}))
    with pytest.raises(ValueError):
        groupby_aggregation(t, [], [("v", "sum", "s")])
    with pytest.raises(ValueError):
        groupby_aggregation(t, ["k"], [("v", "not_an_agg", "s")])
    with pytest.raises(ValueError):
        groupby_aggregation(t, ["k"], [("v", "count_all", "s")])
    with pytest.raises(ValueError):
        groupby_aggregation(t, ["k"], [("v", "sum", "k")])
    with pytest.raises(TypeError):
        groupby_aggregation(t, ["k"], [("v", ("sum", 3), "s")])


def test_columns_roundtrip_on_host():
    # legate layout conversion (bool masks, Rect<1> ranges) without a device
    rng = np.random.default_rng(0)
    t = pa.table({
        "i": pa.array(rng.integers(-5, 5, 50), mask=rng.random(50) < 0.2),
        "f": pa.array(rng.normal(size=50).astype(np.float32)),
        "s": pa.array([None if i % 7 == 0 else "x" * (i % 5) + str(i) for i in range(50)]),
        "b": pa.array([bool(i % 3) for i in range(50)]),
        "ts": pa.array(np.arange(50, dtype=np.int64), type=pa.timestamp("us")),
    })
    lt = _cpu_table(t)
    assert lt.get_column("i").nullable() and not lt.get_column("f").nullable()
    back = lt.to_arrow()
    assert back.equals(t)
    # slices keep their offsets right
    t2 = t.slice(7, 20)
    assert _cpu_table(t2).to_arrow().equals(t2)


def test_python_distinct_argument_errors():
    from legate_dataframe.lib.stream_compaction import distinct

    tbl = _cpu_table(pa.table({"a": [0, 1, 1], "b": [1.0, 2.0, 3.0]}))
    with pytest.raises(ValueError):
        distinct(tbl, [])
    with pytest.raises(IndexError):
        distinct(tbl, ["nope"])


def test_arrow_conversion_argument_errors_without_gpu():
    L = N.lib()
    assert L.ldf_b200_arrow_offsets_to_ranges(None, 3, 4, None, None) == N.LDF_ERR_INVALID_ARGUMENT
    assert b"4 or 8 bytes" in L.ldf_b200_last_error()
    assert L.ldf_b200_arrow_bits_to_bytes(None, 0, -1, None, None) == N.LDF_ERR_INVALID_ARGUMENT
    assert L.ldf_b200_arrow_bits_to_bytes(None, 0, 0, None, None) == N.LDF_OK  # nothing to do
