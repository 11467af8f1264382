"""The reference's CPU task bodies restated with pyarrow -- TEST INFRASTRUCTURE
and CPU BASELINE ONLY (see ``oracle/__init__.py``).

legate-dataframe's ``cpu_variant`` tasks are thin drivers of Arrow C++ (Acero
hashjoin / aggregate and compute SortIndices + Take).  The same Arrow calls,
with the same pre-processing, are made here through pyarrow (Arrow C++ 24.0 in
this image; the reference pins 19.0.*).  ``use_threads=False`` is exactly one
legate CPU task; ``use_threads=True`` lets Acero use every host core.
"""

from __future__ import annotations

import pyarrow as pa
import pyarrow.acero as acero
import pyarrow.compute as pc

_JOIN_TYPES = {
    "inner": "inner",
    "left": "left outer",
    "full": "full outer",
    "semi": "left semi",
    "anti": "left anti",
}


def _default_scalar(t: pa.DataType):
    # create_default_value_scalar (cpp/src/join.cpp:99-109): 0, or "" for strings
    if pa.types.is_string(t) or pa.types.is_large_string(t):
        return pa.scalar("", type=t)
    if pa.types.is_boolean(t):
        return pa.scalar(False)
    return pa.scalar(0, type=t) if not (pa.types.is_timestamp(t) or pa.types.is_date(t)) else pa.scalar(0, type=pa.int64()).cast(t)


def _process_key_column(table: pa.Table, key: str, has_nulls: bool, needs_masks: bool, fields: list):
    """process_key_column (cpp/src/join.cpp:117-162): coalesce a nullable key
    and add its validity as an extra boolean key."""
    col = table.column(key)
    if not has_nulls:
        fields.append(key)
    else:
        replaced = pc.coalesce(col, _default_scalar(col.type))
        table = table.append_column(key + "_replaced", replaced)
        fields.append(key + "_replaced")
    if not needs_masks:
        return table
    table = table.append_column(key + "_mask", pc.is_valid(col))
    fields.append(key + "_mask")
    return table


def join(lhs: pa.Table, rhs: pa.Table, lhs_keys, rhs_keys, join_type: str, nulls_equal: bool = True,
         lhs_out=None, rhs_out=None, use_threads: bool = False) -> pa.Table:
    """arrow_join_and_gather (cpp/src/join.cpp:168-228)."""
    lhs_out = list(lhs.column_names) if lhs_out is None else list(lhs_out)
    if rhs_out is None:
        rhs_out = [] if join_type in ("semi", "anti") else list(rhs.column_names)
    lt, rt = lhs, rhs
    lf, rf = [], []
    if not nulls_equal:
        lf, rf = list(lhs_keys), list(rhs_keys)
    else:
        for lk, rk in zip(lhs_keys, rhs_keys):
            ln = lhs.column(lk).null_count > 0
            rn = rhs.column(rk).null_count > 0
            lt = _process_key_column(lt, lk, ln, ln or rn, lf)
            rt = _process_key_column(rt, rk, rn, ln or rn, rf)
    opts = acero.HashJoinNodeOptions(
        _JOIN_TYPES[join_type], lf, rf, left_output=lhs_out,
        right_output=rhs_out if join_type not in ("semi", "anti") else None,
        output_suffix_for_left="_left", output_suffix_for_right="_right",
    )
    decl = acero.Declaration(
        "hashjoin", opts,
        inputs=[acero.Declaration("table_source", acero.TableSourceNodeOptions(lt)),
                acero.Declaration("table_source", acero.TableSourceNodeOptions(rt))],
    )
    res = decl.to_table(use_threads=use_threads)
    if join_type in ("semi", "anti"):
        # Acero keeps every lhs column (helper key columns included) here
        return pa.Table.from_arrays([res.column(c) for c in lhs_out], names=lhs_out)
    return pa.Table.from_arrays(res.columns, names=lhs_out + rhs_out)


def groupby(table: pa.Table, keys, aggs, use_threads: bool = False) -> pa.Table:
    """GroupByAggregationTask::cpu_variant (cpp/src/groupby_aggregation.cpp:41-94):
    Acero `aggregate` with hash_<kind>; aggs are (in_col|None, kind|(kind, opts), out_name)."""
    reqs = []
    for in_col, kind, _ in aggs:
        if isinstance(kind, tuple):
            k, opts = kind
            reqs.append((in_col, k, opts))
        elif kind == "count_all":
            reqs.append(([], "count_all"))
        else:
            reqs.append((in_col, kind))
    res = pa.TableGroupBy(table, list(keys), use_threads=use_threads).aggregate(reqs)
    # Acero puts the aggregates first, then the keys; legate's output order is
    # keys then aggregates (groupby_aggregation.cpp:166-190)
    nagg = len(aggs)
    cols = list(res.columns)
    if res.column_names[: len(keys)] == list(keys):
        key_cols, agg_cols = cols[: len(keys)], cols[len(keys):]
    else:
        agg_cols, key_cols = cols[:nagg], cols[nagg:]
    return pa.Table.from_arrays(key_cols + agg_cols, names=list(keys) + [a[2] for a in aggs])


def sort(table: pa.Table, keys, ascending=None, nulls_at_end=True, limit=None) -> pa.Table:
    """SortTask::cpu_variant (cpp/src/sort.cpp:312-343): SortIndices + Take,
    one null placement for all keys, then apply_limit."""
    ascending = [True] * len(keys) if ascending is None else list(ascending)
    sk = [(k, "ascending" if a else "descending") for k, a in zip(keys, ascending)]
    idx = pc.sort_indices(table, sort_keys=sk, null_placement="at_end" if nulls_at_end else "at_start")
    out = table.take(idx)
    if limit is not None and abs(limit) < out.num_rows:
        out = out.slice(out.num_rows + limit, -limit) if limit < 0 else out.slice(0, limit)
    return out
