"""LogicalTable: named device-resident columns (mirror of legate-dataframe's
LogicalTable, cpp/include/legate_dataframe/core/table.hpp:49-341 and
python/legate_dataframe/lib/core/table.pyx)."""

from __future__ import annotations

from typing import Iterable

import pyarrow as pa

from legate_dataframe.lib.core.column import LogicalColumn


class LogicalTable:
    def __init__(self, columns: Iterable[LogicalColumn], column_names: Iterable[str]):
        self._columns = list(columns)
        self._names = [str(n) for n in column_names]
        if len(self._columns) != len(self._names):
            raise ValueError("number of columns and column names differ")
        if len(set(self._names)) != len(self._names):
            raise ValueError("column names must be unique")
        if self._columns:
            n = self._columns[0].num_rows()
            if any(c.num_rows() != n for c in self._columns):
                raise ValueError("all columns must have the same number of rows")

    @staticmethod
    def from_arrow(table: pa.Table, device=None) -> "LogicalTable":
        columns = [LogicalColumn.from_arrow(a.combine_chunks(), device) for a in table.columns]
        return LogicalTable(columns, table.column_names)

    def to_arrow(self) -> pa.Table:
        return pa.Table.from_arrays([c.to_arrow() for c in self._columns], names=self._names)

    def num_columns(self) -> int:
        return len(self._columns)

    def num_rows(self) -> int:
        return self._columns[0].num_rows() if self._columns else 0

    def get_column_names(self) -> list[str]:
        return list(self._names)

    def get_column_name_to_index(self) -> dict[str, int]:
        return {n: i for i, n in enumerate(self._names)}

    def get_column(self, key) -> LogicalColumn:
        if isinstance(key, str):
            try:
                key = self._names.index(key)
            except ValueError:
                raise KeyError(key) from None
        return self._columns[key]

    def __getitem__(self, key) -> LogicalColumn:
        return self.get_column(key)

    def get_columns(self) -> list[LogicalColumn]:
        return list(self._columns)

    def select(self, names: Iterable) -> "LogicalTable":
        names = list(names)
        cols = [self.get_column(n) for n in names]
        out_names = [n if isinstance(n, str) else self._names[n] for n in names]
        return LogicalTable(cols, out_names)

    def __repr__(self) -> str:
        cols = ", ".join(f"{n}: {c.arrow_type}" for n, c in zip(self._names, self._columns))
        return f"LogicalTable(rows={self.num_rows()}, {cols})"
