"""csv_read / csv_write: mirror of legate::dataframe::csv_read and csv_write
(python/legate_dataframe/lib/csv.pyx:40-150, cpp/src/csv.cpp, cpp/src/csv.cu).

Columns of Boolean, integer, floating-point and string types are parsed on the
device (``ldf_b200_csv_read``, csrc/csv.cu): each file's bytes are copied to
the GPU as they are and split into records, converted and laid out in the
legate layout there, with the conversions of the reference's CPU reader
(Arrow's CSV reader: its null spellings, quoting, whitespace trimming of
numbers, 0x-hex integers, correctly rounded floats, UTF-8 checks).  A read
that asks for another type (timestamps, dates) is parsed on the host by Arrow
and moved to the device with `LogicalTable.from_arrow`.  Several files are
read one after another and concatenated on the device, as the reference
concatenates its per-file tables.  A table is one partition here, so
`csv_write` writes ``part.0.csv`` into the directory."""

from __future__ import annotations

import ctypes
import io
import os
import pathlib

import numpy as np
import pyarrow as pa
import pyarrow.csv as pacsv
import torch

from legate_dataframe import _native as N
from legate_dataframe.lib.core.column import LogicalColumn, ldf_type_of
from legate_dataframe.lib.core.table import LogicalTable
from legate_dataframe.lib.parquet import _file_list, _file_to_device


def _parsed_on_device(t: pa.DataType) -> bool:
    return (pa.types.is_boolean(t) or pa.types.is_integer(t) or t in (pa.float32(), pa.float64())
            or pa.types.is_string(t) or pa.types.is_large_string(t))

# Arrow's default null spellings (ConvertOptions.null_values), used when na_filter is on
_NULL_SPELLINGS = list(pacsv.ConvertOptions().null_values)


def _arrow_type(d) -> pa.DataType:
    if isinstance(d, pa.DataType):
        return d
    if isinstance(d, str):
        return pa.type_for_alias(d)
    return pa.from_numpy_dtype(np.dtype(d))


def _first_record(path, delimiter: str) -> bytes:
    """The first non-empty record of a file (the header), found with the same
    quoting rules as the device reader."""
    delim = delimiter.encode()
    with open(path, "rb") as f:
        data = b""
        while True:
            block = f.read(1 << 16)
            data += block
            start, i, state = 0, 0, 0  # 0 field start, 1 unquoted, 2 quoted, 3 after a quote in quotes
            while i < len(data):
                c = data[i:i + 1]
                term = c == b"\n" or (c == b"\r" and data[i + 1:i + 2] != b"\n" and (i + 1 < len(data) or not block))
                if state == 2:
                    state = 3 if c == b'"' else 2
                elif c == b'"' and state in (0, 3):
                    state = 2
                elif c == delim:
                    state = 0
                elif term:
                    rec = data[start:i].rstrip(b"\r") if c == b"\n" else data[start:i]
                    if rec:
                        return rec
                    start, state = i + 1, 0
                elif c != b"\r":
                    state = 1
                i += 1
            if not block:
                return data[start:]


def _header_names(path, delimiter: str) -> list[str]:
    rec = _first_record(path, delimiter)
    if not rec:
        return []
    return pacsv.read_csv(io.BytesIO(rec + b"\n"), parse_options=pacsv.ParseOptions(delimiter=delimiter)).schema.names


def _read_file_device(path, fields, types, header: bool, na_filter: bool, delimiter: str) -> list[LogicalColumn]:
    dev = N.require_cuda()
    L = N.lib()
    _, text, size = _file_to_device(path, dev)
    nulls = _NULL_SPELLINGS if na_filter else []
    blob = b"".join(s.encode() + b"\0" for s in nulls)
    ldf_types = [ldf_type_of(t) for t in types]
    alloc = N.TorchAllocator(dev)
    out = (N.ldf_column * len(types))()
    nrows = ctypes.c_int64(0)
    status = L.ldf_b200_csv_read(
        text.data_ptr(), size, delimiter.encode(), 1 if header else 0, N.int32_array(fields),
        N.int32_array(ldf_types), len(types), blob, len(blob), len(nulls), out, ctypes.byref(nrows),
        ctypes.byref(alloc.struct), ctypes.c_void_p(N.current_stream_handle()))
    N.check(status)  # the call has finished with `text` when it returns
    return [LogicalColumn.from_c(out[j], types[j], alloc) for j in range(len(types))]


def _concat(parts: list[list[LogicalColumn]]) -> list[LogicalColumn]:
    """Per-file columns of the same types, end to end on the device."""
    if len(parts) == 1:
        return parts[0]
    cols = []
    for j, first in enumerate(parts[0]):
        pieces = [p[j] for p in parts]
        n = sum(c.size for c in pieces)
        w = N.TYPE_WIDTH[first.ldf_type]
        dev = first.data.device
        valid = None
        if any(c.valid is not None for c in pieces):
            valid = torch.cat([c.valid[:c.size] if c.valid is not None else torch.ones(c.size, dtype=torch.uint8,
                                                                                        device=dev) for c in pieces])
        if first.ldf_type == N.LDF_STRING:
            ranges, chars, base = [], [], 0
            for c in pieces:
                r = c.data[: 16 * c.size].view(torch.int64).view(c.size, 2) - c.chars_base + base
                ranges.append(r.reshape(-1))
                chars.append(c.chars[: c.num_chars])
                base += c.num_chars
            data = torch.cat(ranges).view(torch.uint8) if n else torch.empty(16, dtype=torch.uint8, device=dev)
            allc = torch.cat(chars) if base else torch.empty(16, dtype=torch.uint8, device=dev)
            cols.append(LogicalColumn(first.arrow_type, first.ldf_type, n, data, valid, allc, 0, base))
        else:
            data = torch.cat([c.data[: w * c.size] for c in pieces]) if n else first.data[:0]
            cols.append(LogicalColumn(first.arrow_type, first.ldf_type, n, data, valid))
    return cols


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
    if not isinstance(delimiter, str) or len(delimiter) != 1 or delimiter in '"\r\n' or ord(delimiter) > 127:
        raise ValueError("delimiter must be one ASCII character other than a quote or a line end")

    if all(_parsed_on_device(t) for t in dtypes) and len(dtypes) <= 64:
        parts = []
        for p in paths:
            if usecols is None:  # header row: select by name
                hdr = _header_names(p, delimiter)
                missing = [n for n in names if n not in hdr]
                if missing and hdr:
                    raise ValueError(f"columns not in the CSV header: {missing}")
                if not hdr:  # empty file: no rows, as the reference skips it
                    continue
                fields = [hdr.index(n) for n in names]
            else:
                fields = usecols
            parts.append(_read_file_device(p, fields, dtypes, usecols is None, na_filter, delimiter))
        if not parts:
            return LogicalTable.from_arrow(pa.table({n: pa.array([], t) for n, t in zip(names, dtypes)}))
        return LogicalTable(_concat(parts), names)

    # other types: Arrow on the host, then the device layout
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
