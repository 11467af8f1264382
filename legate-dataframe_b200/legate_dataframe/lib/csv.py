"""csv_read / csv_write: mirror of legate::dataframe::csv_read and csv_write
(python/legate_dataframe/lib/csv.pyx:40-150, cpp/src/csv.cpp).

Files are parsed on the host by Arrow's CSV reader into the requested types;
the columns then go to the device in the legate layout through
`LogicalTable.from_arrow` (Arrow buffers copied as they are, validity
bitmaps and string offsets expanded on the device).  A table is one
partition here, so `csv_write` writes ``part.0.csv`` into the directory."""

from __future__ import annotations

import pathlib

import numpy as np
import pyarrow as pa
import pyarrow.csv as pacsv

from legate_dataframe.lib.core.table import LogicalTable
from legate_dataframe.lib.parquet import _file_list


def _arrow_type(d) -> pa.DataType:
    if isinstance(d, pa.DataType):
        return d
    if isinstance(d, str):
        return pa.type_for_alias(d)
    return pa.from_numpy_dtype(np.dtype(d))


def csv_read(files, *, dtypes, na_filter=True, delimiter=",", usecols=None, names=None) -> LogicalTable:
    """Read CSV files into a logical table.

    ``dtypes``: the Arrow type of each read column (or one type for all).
    ``usecols``: column names to read (the file has a header); as integers the
    file has no header and ``names`` names them.  ``names`` without
    ``usecols`` names the header columns to read.  ``na_filter=False`` reads
    no nulls (empty fields stay empty strings / fail for numbers)."""
    paths = _file_list(files)
    if not paths:
        raise ValueError("no files to read")
    if names is None:
        names, usecols = usecols, None  # usecols must then be column names
    if names is None:
        raise ValueError("pass the column names (usecols or names)")
    names = list(names)
    if usecols is not None:
        usecols = list(usecols)
        if len(usecols) != len(names) or not all(isinstance(u, int) for u in usecols):
            raise ValueError("integral usecols must match names in length")
    if isinstance(dtypes, (pa.DataType, str)):
        dtypes = [dtypes] * len(names)
    dtypes = [_arrow_type(d) for d in dtypes]
    if len(dtypes) != len(names):
        raise ValueError("dtypes must match the read columns in length")

    if usecols is None:  # header row: select by name
        read_opts = pacsv.ReadOptions()
        include = names
        rename = None
    else:  # no header: generated names f0, f1, ...
        read_opts = pacsv.ReadOptions(autogenerate_column_names=True)
        include = [f"f{i}" for i in usecols]
        rename = names
    conv = pacsv.ConvertOptions(column_types=dict(zip(include, dtypes)), include_columns=include,
                                strings_can_be_null=na_filter, quoted_strings_can_be_null=na_filter)
    if not na_filter:
        conv.null_values = []
    parse = pacsv.ParseOptions(delimiter=delimiter)
    tables = [pacsv.read_csv(p, read_options=read_opts, parse_options=parse, convert_options=conv) for p in paths]
    table = tables[0] if len(tables) == 1 else pa.concat_tables(tables)
    if rename is not None:
        table = table.rename_columns(rename)
    return LogicalTable.from_arrow(table)


def csv_write(tbl: LogicalTable, path, delimiter=",") -> None:
    """Write the table to ``path/part.0.csv`` (the directory is created)."""
    out = pathlib.Path(path)
    out.mkdir(parents=True, exist_ok=True)
    pacsv.write_csv(tbl.to_arrow(), out / "part.0.csv", write_options=pacsv.WriteOptions(delimiter=delimiter))
