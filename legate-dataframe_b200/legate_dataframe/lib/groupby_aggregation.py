"""groupby_aggregation(): mirror of
python/legate_dataframe/lib/groupby_aggregation.pyx:48-117 and the C++
``legate::dataframe::groupby_aggregation`` (cpp/src/groupby_aggregation.cpp:135-232),
running the sm_100a hash aggregation of libldf_b200.so."""

from __future__ import annotations

import ctypes
from typing import Iterable, Tuple

import pyarrow as pa
import pyarrow.compute as pc

from legate_dataframe import _native as N
from legate_dataframe.lib.core.column import LogicalColumn, ldf_type_of
from legate_dataframe.lib.core.table import LogicalTable

# Aggregations of the B200 path (the Arrow function names the reference takes).
SUPPORTED = ("sum", "min", "max", "count", "count_all", "mean", "count_distinct")
# Accepted by the reference but outside this path's kernels.
KNOWN = SUPPORTED + ("product", "variance", "stddev", "approximate_median")


def _strip_hash(kind: str) -> str:
    return kind[5:] if kind.startswith("hash_") else kind


_OUTPUT_TYPES: dict = {}


def _output_type(values_type: pa.DataType, kind: str, options) -> pa.DataType:
    """Output type = the Arrow hash_<kind> result type, found with a dummy
    aggregation on empty input exactly like make_output_column
    (groupby_aggregation.cpp:100-132).  The answer depends only on the value
    type, the kind and the options, so it is computed once per combination
    (the dummy aggregation costs about 0.1 ms, as much as a small groupby)."""
    if kind in ("count_all", "count_distinct"):
        return pa.int64()
    key = (str(values_type), kind, None if options is None else (type(options).__name__, str(options)))
    hit = _OUTPUT_TYPES.get(key)
    if hit is not None:
        return hit
    _OUTPUT_TYPES[key] = t = _dummy_output_type(values_type, kind, options)
    return t


def _dummy_output_type(values_type: pa.DataType, kind: str, options) -> pa.DataType:
    tbl = pa.table({"keys": pa.array([], pa.int32()), "values": pa.array([], values_type)})
    agg = ("values", kind, options) if options is not None else ("values", kind)
    res = pa.TableGroupBy(tbl, "keys").aggregate([agg])
    return res.schema.field(f"values_{kind}").type


def _count_mode(options) -> int:
    if options is None:
        return N.LDF_COUNT_ONLY_VALID
    if not isinstance(options, pc.CountOptions):
        raise ValueError("Options are not supported for this aggregation")
    mode = str(options).split("mode=")[-1].rstrip(")").strip().upper()
    if mode == "NULLS":
        return N.LDF_COUNT_ONLY_NULL
    if mode == "ALL":
        return N.LDF_COUNT_ALL
    return N.LDF_COUNT_ONLY_VALID


def groupby_aggregation(
    table: LogicalTable,
    keys: Iterable[str],
    column_aggregations: Iterable[Tuple[str, str, str]],
) -> LogicalTable:
    """Group ``table`` by ``keys`` and aggregate.

    ``column_aggregations`` holds ``(input column, kind, output name)`` with
    kind one of "sum", "min", "max", "count", "count_all", "mean",
    "count_distinct", or ``(kind, pyarrow.compute.CountOptions)`` for the
    count kinds.  The output holds the key columns then one column per
    aggregation in request order; row order is unspecified.  Null keys form a
    group.  The table's columns may be device tensors or host tensors (pinned
    for full copy speed): host columns are copied to the device inside the
    call, overlapped with the passes that do not need them yet.
    """
    keys = list(keys)
    if len(keys) == 0:
        raise ValueError("must pass at least one key column")
    names = table.get_column_name_to_index()
    for k in keys:
        if k not in names:
            raise ValueError(f"unknown key column: {k}")

    aggs = []
    out_names = list(keys)
    out_types = []
    for in_col_name, kind, out_col_name in column_aggregations:
        options = None
        if isinstance(kind, tuple):
            kind, options = kind
            if not isinstance(options, pc.FunctionOptions):
                raise TypeError("options must be an arrow `FunctionOptions` object.")
        if not isinstance(kind, str):
            raise TypeError("aggregation kind must be string or tuple of string and options.")
        kind = _strip_hash(kind)
        if kind not in KNOWN:
            raise ValueError(f"unknown aggregation function: {kind}")
        if kind not in SUPPORTED:
            raise ValueError(f"aggregation '{kind}' is not supported by the B200 groupby path")
        if kind == "count_all":
            if in_col_name is not None:
                raise ValueError("input column name must be `None` for 'count_all'")
            if options is not None:
                raise ValueError("count_all does not support options")
            in_idx = names[keys[0]]
            mode = N.LDF_COUNT_ALL
        else:
            if in_col_name not in names:
                raise ValueError(f"unknown input column: {in_col_name}")
            in_idx = names[in_col_name]
            if kind in ("count", "count_distinct"):
                mode = _count_mode(options)
            elif options is not None:
                raise ValueError("Options are not supported for this aggregation")
            else:
                mode = N.LDF_COUNT_ONLY_VALID
        if out_col_name in out_names:
            raise ValueError("name conflict in the output columns: " + out_col_name)
        out_names.append(out_col_name)
        values_type = table.get_column(in_idx).arrow_type
        otype = _output_type(values_type, kind, options)
        out_types.append(otype)
        aggs.append(N.ldf_aggregation(in_idx, N.LDF_AGG[kind], mode, ldf_type_of(otype)))

    dev = N.require_cuda()
    L = N.lib()
    alloc = N.TorchAllocator(dev)
    cols = (N.ldf_column * max(table.num_columns(), 1))(*[c.to_c() for c in table.get_columns()])
    key_idx = [names[k] for k in keys]
    nout = len(keys) + len(aggs)
    out = (N.ldf_column * nout)()
    agg_arr = (N.ldf_aggregation * max(len(aggs), 1))(*aggs)
    status = L.ldf_b200_groupby_aggregation(
        cols, table.num_columns(), N.int32_array(key_idx), len(key_idx), agg_arr, len(aggs), out,
        ctypes.byref(alloc.struct), ctypes.c_void_p(N.current_stream_handle()),
    )
    N.check(status)
    types = [table.get_column(i).arrow_type for i in key_idx] + out_types
    res = [LogicalColumn.from_c(out[j], types[j], alloc) for j in range(nout)]
    return LogicalTable(res, out_names)
