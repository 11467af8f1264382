"""join(): mirror of python/legate_dataframe/lib/join.pyx:53-146 and the C++
``legate::dataframe::join`` (cpp/src/join.cpp:328-477), running the sm_100a
hash join of libldf_b200.so (``ldf_b200_join``)."""

from __future__ import annotations

import ctypes
from enum import IntEnum
from typing import Iterable, Optional

from legate_dataframe import _native as N
from legate_dataframe.lib.core.column import LogicalColumn
from legate_dataframe.lib.core.table import LogicalTable


class JoinType(IntEnum):
    """Options for the join type (``INNER``, ``LEFT``, ``FULL``, ``SEMI``, ``ANTI``)."""

    INNER = 0
    LEFT = 1
    FULL = 2
    SEMI = 3
    ANTI = 4


class BroadcastInput(IntEnum):
    """Options for input broadcasting (``AUTO``, ``LEFT``, and ``RIGHT``)."""

    AUTO = 0
    LEFT = 1
    RIGHT = 2


def join(
    lhs: LogicalTable,
    rhs: LogicalTable,
    *,
    lhs_keys: Iterable[str],
    rhs_keys: Iterable[str],
    join_type: JoinType,
    lhs_out_columns: Optional[Iterable[str]] = None,
    rhs_out_columns: Optional[Iterable[str]] = None,
    nulls_equal: bool = True,
    broadcast: BroadcastInput = BroadcastInput.AUTO,
) -> LogicalTable:
    """Hash join of two tables (build on ``rhs``, probe with ``lhs``).

    Output: the ``lhs_out_columns`` then the ``rhs_out_columns`` (all columns
    by default; none of ``rhs`` for SEMI/ANTI).  LEFT makes the rhs columns
    nullable and FULL every column.  Row order is unspecified.

    Raises ValueError when the key lists differ in length, output names
    collide or SEMI/ANTI select rhs columns; RuntimeError for a forced
    broadcast that needs repartitioning (join.cpp:386-396).
    """
    join_type = JoinType(join_type)
    broadcast = BroadcastInput(broadcast)
    lhs_keys = list(lhs_keys)
    rhs_keys = list(rhs_keys)
    if lhs_out_columns is None:
        lhs_out_columns = lhs.get_column_names()
    if rhs_out_columns is None:
        if join_type in (JoinType.ANTI, JoinType.SEMI):
            rhs_out_columns = []
        else:
            rhs_out_columns = rhs.get_column_names()
    lhs_out_columns = list(lhs_out_columns)
    rhs_out_columns = list(rhs_out_columns)

    if len(lhs_keys) != len(rhs_keys):
        raise ValueError("The size of `lhs_keys` and `rhs_keys` must be equal")
    if join_type in (JoinType.SEMI, JoinType.ANTI) and rhs_out_columns:
        raise ValueError("rhs must have no output columns for SEMI and ANTI join")
    if broadcast != BroadcastInput.AUTO and (
        join_type == JoinType.FULL or (broadcast == BroadcastInput.LEFT and join_type != JoinType.INNER)
    ):
        raise RuntimeError(
            "Force broadcast was indicated, but repartitioning is required. "
            "FULL joins do not support broadcasting and LEFT/SEMI/ANTI joins only for the "
            "right hand side argument."
        )
    out_names = lhs_out_columns + rhs_out_columns
    if len(set(out_names)) != len(out_names):
        raise ValueError("column names of the join result must be unique")

    lidx = lhs.get_column_name_to_index()
    ridx = rhs.get_column_name_to_index()
    try:
        lk = [lidx[k] for k in lhs_keys]
        rk = [ridx[k] for k in rhs_keys]
        lo = [lidx[k] for k in lhs_out_columns]
        ro = [ridx[k] for k in rhs_out_columns]
    except KeyError as e:
        raise ValueError(f"unknown column name {e}") from None
    for a, b in zip(lk, rk):
        if lhs.get_column(a).arrow_type != rhs.get_column(b).arrow_type:
            raise ValueError("join key types of lhs and rhs must match")

    dev = N.require_cuda()
    L = N.lib()
    alloc = N.TorchAllocator(dev)
    lcols = (N.ldf_column * max(lhs.num_columns(), 1))(*[c.to_c() for c in lhs.get_columns()])
    rcols = (N.ldf_column * max(rhs.num_columns(), 1))(*[c.to_c() for c in rhs.get_columns()])
    nout = len(lo) + len(ro)
    out = (N.ldf_column * max(nout, 1))()
    status = L.ldf_b200_join(
        lcols, lhs.num_columns(), rcols, rhs.num_columns(),
        N.int32_array(lk), N.int32_array(rk), len(lk), int(join_type), 1 if nulls_equal else 0,
        N.int32_array(lo), len(lo), N.int32_array(ro), len(ro),
        out, ctypes.byref(alloc.struct), ctypes.c_void_p(N.current_stream_handle()),
    )
    N.check(status)
    types = [lhs.get_column(i).arrow_type for i in lo] + [rhs.get_column(i).arrow_type for i in ro]
    cols = [LogicalColumn.from_c(out[j], types[j], alloc) for j in range(nout)]
    return LogicalTable(cols, out_names)
