"""LogicalTable: named device-resident columns (mirror of legate-dataframe's
LogicalTable, cpp/include/legate_dataframe/core/table.hpp:49-341 and
python/legate_dataframe/lib/core/table.pyx)."""

from __future__ import annotations

from typing import Iterable

import pyarrow as pa
import torch

from legate_dataframe import _native as N
from legate_dataframe.lib.core.column import LogicalColumn

_BITS = None


def _pack_bits(u8: torch.Tensor) -> torch.Tensor:
    """One byte per row (nonzero = set) -> an Arrow LSB-first bitmap, on the device."""
    global _BITS
    n = u8.numel()
    nb = (n + 7) // 8
    b = (u8 != 0).to(torch.uint8)
    if nb * 8 != n:
        b = torch.nn.functional.pad(b, (0, nb * 8 - n))
    if _BITS is None or _BITS.device != u8.device:
        _BITS = torch.tensor([1, 2, 4, 8, 16, 32, 64, 128], dtype=torch.uint8, device=u8.device)
    return (b.view(nb, 8) * _BITS).sum(dim=1, dtype=torch.uint8)


def _device_fixed(c: LogicalColumn) -> bool:
    return c.ldf_type != N.LDF_STRING and c.data is not None and c.data.is_cuda


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
        """Copy to a host Arrow table.  Fixed-width device columns go through
        one pinned staging buffer: validity (and bool values) are bit-packed on
        the device, every buffer is copied asynchronously, the stream is
        synchronized once, and the Arrow arrays wrap the staging memory
        without another copy."""
        arrays = [None] * len(self._columns)
        pieces = []  # (column index, role, device uint8 tensor)
        nulls = []
        for i, c in enumerate(self._columns):
            if not _device_fixed(c) or c.size == 0:
                continue
            n, w = c.size, N.TYPE_WIDTH[c.ldf_type]
            data = c.data[: n * w]
            pieces.append((i, "data", _pack_bits(data) if c.ldf_type == N.LDF_BOOL8 else data))
            if c.valid is not None:
                v = c.valid[:n]
                pieces.append((i, "valid", _pack_bits(v)))
                nulls.append((i, (v == 0).sum()))
        if pieces:
            counts = torch.stack([t for _, t in nulls]).to(torch.int64).view(torch.uint8) if nulls else None
            offs, total = [], 0
            for _, _, t in pieces:
                offs.append(total)
                total += (t.numel() + 63) & ~63
            if counts is not None:
                count_off = total
                total += counts.numel()
            host = torch.empty(max(total, 1), dtype=torch.uint8, pin_memory=True)
            for (_, _, t), o in zip(pieces, offs):
                host[o:o + t.numel()].copy_(t, non_blocking=True)
            if counts is not None:
                host[count_off:count_off + counts.numel()].copy_(counts, non_blocking=True)
            torch.cuda.current_stream(pieces[0][2].device).synchronize()
            hnp = host.numpy()
            null_count = {}
            if counts is not None:
                nc = hnp[count_off:count_off + counts.numel()].view("int64")
                null_count = {i: int(x) for (i, _), x in zip(nulls, nc)}
            bufs = {}
            for (i, role, t), o in zip(pieces, offs):
                bufs[(i, role)] = pa.py_buffer(hnp[o:o + t.numel()])
            for i, c in enumerate(self._columns):
                if (i, "data") not in bufs:
                    continue
                typ = pa.bool_() if c.ldf_type == N.LDF_BOOL8 else c.arrow_type
                arrays[i] = pa.Array.from_buffers(typ, c.size, [bufs.get((i, "valid")), bufs[(i, "data")]],
                                                  null_count=null_count.get(i, 0))
        for i, c in enumerate(self._columns):
            if arrays[i] is None:
                arrays[i] = c.to_arrow()
        return pa.Table.from_arrays(arrays, names=self._names)

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
