"""distinct(): mirror of legate::dataframe::distinct
(cpp/include/legate_dataframe/stream_compaction.hpp, cpp/src/stream_compaction.cpp:121-150;
python binding python/legate_dataframe/lib/stream_compaction.pyx).

One row per distinct combination of the key columns, with every column of
the input; for columns that are not keys any value of the group is possible
(the rows here are whole representative rows).  Null keys form one group.
Row order is unspecified.  ``high_cardinality`` only steers the reference's
multi-rank plan (a local distinct before the shuffle); on one GPU it has no
effect and is accepted for API compatibility."""

from __future__ import annotations

from typing import Iterable

from legate_dataframe import _native as N
from legate_dataframe.lib.core.column import LogicalColumn
from legate_dataframe.lib.core.table import LogicalTable


def distinct(tbl: LogicalTable, keys: Iterable[str], high_cardinality: bool = True) -> LogicalTable:
    keys = list(keys)
    if not keys:
        raise ValueError("must pass at least one key column")
    names = tbl.get_column_name_to_index()
    for k in keys:
        if k not in names:
            # std::map::at in the reference (stream_compaction.cpp:130) -> std::out_of_range
            raise IndexError(f"unknown key column: {k}")
    dev = N.require_cuda()
    L = N.lib()
    alloc = N.TorchAllocator(dev)
    ncols = tbl.num_columns()
    cols = (N.ldf_column * max(ncols, 1))(*[c.to_c() for c in tbl.get_columns()])
    out = (N.ldf_column * max(ncols, 1))()
    import ctypes

    status = L.ldf_b200_distinct(cols, ncols, N.int32_array([names[k] for k in keys]), len(keys), out,
                                 ctypes.byref(alloc.struct), ctypes.c_void_p(N.current_stream_handle()))
    N.check(status)
    res = [LogicalColumn.from_c(out[j], tbl.get_column(j).arrow_type, alloc) for j in range(ncols)]
    return LogicalTable(res, tbl.get_column_names())
