"""sort(): mirror of python/legate_dataframe/lib/sort.pyx:30-90 and the C++
``legate::dataframe::sort`` (cpp/src/sort.cpp:379-433), running the sm_100a
onesweep radix sort of libldf_b200.so."""

from __future__ import annotations

import ctypes

from legate_dataframe import _native as N
from legate_dataframe.lib.core.column import LogicalColumn
from legate_dataframe.lib.core.table import LogicalTable

INT64_MIN = -(2**63)


def sort(
    tbl: LogicalTable,
    keys: list,
    *,
    sort_ascending: list = None,
    nulls_at_end=True,
    stable=False,
    limit=None,
) -> LogicalTable:
    """Sort the table by ``keys`` (lexicographic, per-key direction).

    ``nulls_at_end`` places nulls last (True) or first, for every key
    regardless of direction.  The result is always the stable order.
    ``limit`` > 0 keeps the first rows, < 0 the last.
    Raises ValueError for empty/unknown/duplicate keys or a
    ``sort_ascending`` of the wrong length (sort.cpp:386-406).
    """
    keys = list(keys) if keys is not None else []
    if len(keys) == 0:
        raise ValueError("must sort along at least one column")
    if sort_ascending is None:
        sort_ascending = [True] * len(keys)
    sort_ascending = [bool(a) for a in sort_ascending]
    if len(sort_ascending) != len(keys):
        raise ValueError("sort column order and null precedence must match number of keys")
    if len(set(keys)) != len(keys):
        raise ValueError("duplicate sort keys")
    names = tbl.get_column_name_to_index()
    for k in keys:
        if k not in names:
            raise ValueError(f"sort key '{k}' not found in table")
    key_idx = [names[k] for k in keys]

    dev = N.require_cuda()
    L = N.lib()
    alloc = N.TorchAllocator(dev)
    cols = (N.ldf_column * max(tbl.num_columns(), 1))(*[c.to_c() for c in tbl.get_columns()])
    asc = (ctypes.c_uint8 * len(keys))(*[1 if a else 0 for a in sort_ascending])
    out = (N.ldf_column * max(tbl.num_columns(), 1))()
    lim = INT64_MIN if limit is None else int(limit)
    status = L.ldf_b200_sort(
        cols, tbl.num_columns(), N.int32_array(key_idx), asc, len(keys), 1 if nulls_at_end else 0,
        1 if stable else 0, lim, out, ctypes.byref(alloc.struct), ctypes.c_void_p(N.current_stream_handle()),
    )
    N.check(status)
    res = [LogicalColumn.from_c(out[j], tbl.get_column(j).arrow_type, alloc) for j in range(tbl.num_columns())]
    return LogicalTable(res, tbl.get_column_names())
