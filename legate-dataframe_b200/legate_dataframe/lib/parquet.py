"""parquet_read / parquet_write: mirror of legate::dataframe::parquet_read and
parquet_write (python/legate_dataframe/lib/parquet.pyx:49-135,
cpp/src/parquet.cpp).

Files are decoded on the host by Arrow's Parquet reader; the columns then go
to the device in the legate layout through `LogicalTable.from_arrow`, which
copies Arrow's buffers as they are and expands the validity bitmaps and
string offsets on the device.  A table is one partition here, so
`parquet_write` writes ``part.0.parquet`` into the directory."""

from __future__ import annotations

import glob
import pathlib

import pyarrow as pa
import pyarrow.parquet as pq

from legate_dataframe.lib.core.table import LogicalTable


def _file_list(files) -> list[str]:
    if isinstance(files, str):
        return sorted(glob.glob(files))
    if isinstance(files, pathlib.Path):
        return [str(files)]
    return [str(f) for f in files]


def parquet_read(files, *, columns=None, ignore_row_groups=None) -> LogicalTable:
    """Read Parquet files into a logical table.

    ``files``: a glob string, a path, or an iterable of paths; their tables
    are concatenated in order.  ``columns`` selects a subset of columns.
    ``ignore_row_groups`` only steers the reference's chunked multi-task read
    and is accepted for API compatibility."""
    paths = _file_list(files)
    if not paths:
        raise ValueError("no files to read")
    cols = None if columns is None else list(columns)
    tables = [pq.read_table(p, columns=cols) for p in paths]
    table = tables[0] if len(tables) == 1 else pa.concat_tables(tables)
    return LogicalTable.from_arrow(table)


def parquet_write(tbl: LogicalTable, path) -> None:
    """Write the table to ``path/part.0.parquet`` (the directory is created)."""
    out = pathlib.Path(path)
    out.mkdir(parents=True, exist_ok=True)
    pq.write_table(tbl.to_arrow(), out / "part.0.parquet")
