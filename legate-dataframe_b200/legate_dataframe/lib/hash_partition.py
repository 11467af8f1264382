"""hash_partition(): the local step of legate-dataframe's
task::repartition_by_hash (cpp/src/core/repartition_by_hash.cu:296-310:
cudf::hash_partition + cudf::split), exposed as a public op.  Rows are
grouped by bucket = hash(keys) % nparts (buckets in order, input order kept
inside a bucket); the bucket start offsets come back with the table."""

from __future__ import annotations

import ctypes
from typing import Iterable

from legate_dataframe import _native as N
from legate_dataframe.lib.core.column import LogicalColumn
from legate_dataframe.lib.core.table import LogicalTable


def hash_partition(tbl: LogicalTable, keys: Iterable[str], nparts: int):
    """Return ``(partitioned_table, offsets)``; ``offsets`` has ``nparts + 1``
    entries, bucket ``b`` being rows ``offsets[b]:offsets[b+1]``."""
    keys = list(keys)
    if not keys:
        raise ValueError("must pass at least one key column")
    if int(nparts) < 1:
        raise ValueError("nparts must be positive")
    names = tbl.get_column_name_to_index()
    for k in keys:
        if k not in names:
            raise ValueError(f"unknown key column: {k}")
    dev = N.require_cuda()
    L = N.lib()
    alloc = N.TorchAllocator(dev)
    cols = (N.ldf_column * max(tbl.num_columns(), 1))(*[c.to_c() for c in tbl.get_columns()])
    out = (N.ldf_column * max(tbl.num_columns(), 1))()
    offsets = (ctypes.c_int64 * (int(nparts) + 1))()
    status = L.ldf_b200_hash_partition(
        cols, tbl.num_columns(), N.int32_array([names[k] for k in keys]), len(keys), int(nparts), out,
        offsets, ctypes.byref(alloc.struct), ctypes.c_void_p(N.current_stream_handle()),
    )
    N.check(status)
    res = [LogicalColumn.from_c(out[j], tbl.get_column(j).arrow_type, alloc) for j in range(tbl.num_columns())]
    return LogicalTable(res, tbl.get_column_names()), list(offsets)
