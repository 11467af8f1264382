"""parquet_read / parquet_write: mirror of legate::dataframe::parquet_read and
parquet_write (python/legate_dataframe/lib/parquet.pyx:49-135,
cpp/src/parquet.cpp, cpp/src/parquet.cu).

Files whose selected columns are flat (optional or required) Boolean,
integer, floating-point, timestamp, date or string columns stored
uncompressed or with Snappy, in PLAIN or dictionary encoding, are decoded on
the device (``ldf_b200_parquet_decode``, csrc/parquet.cu): the file's bytes
are copied to the GPU as they are, the footer and page headers (a few bytes
per page) are read here, and the pages are decompressed and decoded into the
legate layout there.  Other files are decoded on the host by Arrow's Parquet
reader and moved to the device with `LogicalTable.from_arrow`.  A table is
one partition here, so `parquet_write` writes ``part.0.parquet`` into the
directory."""

from __future__ import annotations

import ctypes
import glob
import os
import pathlib
from concurrent.futures import ThreadPoolExecutor, as_completed

import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq
import torch

from legate_dataframe import _native as N
from legate_dataframe.lib.core.table import LogicalTable


def _file_list(files) -> list[str]:
    if isinstance(files, str):
        return sorted(glob.glob(files))
    if isinstance(files, pathlib.Path):
        return [str(files)]
    return [str(f) for f in files]


_READ_PIECE = 64 << 20  # bytes per read (and per host-to-device copy) of a large file


def _file_to_device(path, dev) -> tuple[torch.Tensor, torch.Tensor, int]:
    """The file's bytes in pinned host memory and on the device.  Large files
    are read in 64 MB pieces by a few threads, each piece copied to the device
    as soon as it has been read, so the reads and the copies overlap."""
    size = os.path.getsize(path)
    host = torch.empty(max(size, 16), dtype=torch.uint8, pin_memory=True)
    text = torch.empty(max(size, 16), dtype=torch.uint8, device=dev)
    if size == 0:
        return host, text, 0
    mv = memoryview(host.numpy())
    pieces = [(a, min(a + _READ_PIECE, size)) for a in range(0, size, _READ_PIECE)]

    def read(piece):
        a, b = piece
        with open(path, "rb") as f:
            f.seek(a)
            got = f.readinto(mv[a:b])
        if got != b - a:
            raise OSError(f"short read of {path}")
        return piece

    if len(pieces) == 1:
        read(pieces[0])
        text[:size].copy_(host[:size], non_blocking=True)
    else:
        with ThreadPoolExecutor(max_workers=min(8, len(pieces))) as ex:
            for fut in as_completed([ex.submit(read, pc) for pc in pieces]):
                a, b = fut.result()
                text[a:b].copy_(host[a:b], non_blocking=True)
    return host, text, size


_PHYSICAL = {"BOOLEAN": N.LDF_PQ_BOOLEAN, "INT32": N.LDF_PQ_INT32, "INT64": N.LDF_PQ_INT64,
             "FLOAT": N.LDF_PQ_FLOAT, "DOUBLE": N.LDF_PQ_DOUBLE, "BYTE_ARRAY": N.LDF_PQ_BYTE_ARRAY}
_CODECS = {"UNCOMPRESSED": N.LDF_PQ_UNCOMPRESSED, "SNAPPY": N.LDF_PQ_SNAPPY}


class _NotOnDevice(Exception):
    """The file needs a feature the device decoder does not have."""


def _ldf_output_type(arrow_type: pa.DataType, physical: int) -> int:
    from legate_dataframe.lib.core.column import ldf_type_of

    if physical == N.LDF_PQ_BYTE_ARRAY and not (pa.types.is_string(arrow_type) or pa.types.is_large_string(arrow_type)):
        raise _NotOnDevice("binary column")
    if pa.types.is_timestamp(arrow_type) and physical != N.LDF_PQ_INT64:
        raise _NotOnDevice("timestamp stored as INT96")
    try:
        return ldf_type_of(arrow_type)
    except ValueError as e:
        raise _NotOnDevice(str(e))


def _page_table(host, md, col_indices, physical):
    """One ldf_parquet_page per page of the selected column chunks: the
    chunks' extents come from the footer (Arrow's metadata reader), their page
    headers are walked by the library on the host (ldf_b200_parquet_pages)."""
    nchunks = md.num_row_groups * len(col_indices)
    i64, i32 = ctypes.c_int64 * max(nchunks, 1), ctypes.c_int32 * max(nchunks, 1)
    start, nbytes, row0 = i64(), i64(), i64()
    column, codec, phys = i32(), i32(), i32()
    k, row_base = 0, 0
    for g in range(md.num_row_groups):
        rg = md.row_group(g)
        for j, ci in enumerate(col_indices):
            cc = rg.column(ci)
            if cc.compression not in _CODECS:
                raise _NotOnDevice(f"codec {cc.compression}")
            start[k] = cc.dictionary_page_offset if cc.dictionary_page_offset else cc.data_page_offset
            nbytes[k] = cc.total_compressed_size
            row0[k], column[k], codec[k], phys[k] = row_base, j, _CODECS[cc.compression], physical[j]
            k += 1
        row_base += rg.num_rows
    L = N.lib()
    buf = np.ascontiguousarray(host, dtype=np.uint8)
    args = (buf.ctypes.data, buf.size, start, nbytes, row0, column, codec, phys, nchunks)
    count = ctypes.c_int32(0)

    def walk(table, cap):
        status = L.ldf_b200_parquet_pages(*args, table, cap, ctypes.byref(count))
        if status == N.LDF_ERR_UNSUPPORTED:
            raise _NotOnDevice(L.ldf_b200_last_error().decode("utf-8", "replace"))
        N.check(status)

    walk(None, 0)  # the page count
    table = (N.ldf_parquet_page * max(count.value, 1))()
    walk(table, count.value)
    return table, count.value


def _column_specs(pf, columns):
    """(names, leaf indices, physical types, output types, nullable flags,
    Arrow types) of the selected columns of a ParquetFile (raises
    _NotOnDevice when a column needs what the device decoder lacks)."""
    schema, arrow_schema = pf.schema, pf.schema_arrow
    names = list(arrow_schema.names) if columns is None else list(columns)
    if len(names) == 0 or len(names) > 64:
        raise _NotOnDevice("column count")
    if len(schema) != len(arrow_schema):
        raise _NotOnDevice("nested schema")
    col_indices, physical, types, nullable, arrow_types = [], [], [], [], []
    for name in names:
        i = arrow_schema.get_field_index(name)
        if i < 0:
            raise KeyError(f"column {name!r} not in the file")
        c = schema.column(i)
        if c.path != name or c.max_repetition_level != 0 or c.max_definition_level > 1:
            raise _NotOnDevice("nested column")
        if c.physical_type not in _PHYSICAL:
            raise _NotOnDevice(f"physical type {c.physical_type}")
        ph = _PHYSICAL[c.physical_type]
        at = arrow_schema.field(i).type
        col_indices.append(i)
        physical.append(ph)
        types.append(_ldf_output_type(at, ph))
        nullable.append(1 if c.max_definition_level == 1 else 0)
        arrow_types.append(at)
    return names, col_indices, physical, types, nullable, arrow_types


def _read_file_device(path, columns):
    """The selected columns of one file decoded on the device (raises
    _NotOnDevice when the file needs what the device decoder lacks)."""
    from legate_dataframe.lib.core.column import LogicalColumn

    pf = pq.ParquetFile(path)
    md = pf.metadata
    names, col_indices, physical, types, nullable, arrow_types = _column_specs(pf, columns)
    dev = N.require_cuda()
    host, text, size = _file_to_device(path, dev)
    pages, npages = _page_table(host.numpy(), md, col_indices, physical)
    L = N.lib()
    alloc = N.TorchAllocator(dev)
    out = (N.ldf_column * len(names))()
    status = L.ldf_b200_parquet_decode(
        text.data_ptr(), size, pages, npages, N.int32_array(physical), N.int32_array(types), N.int32_array(nullable),
        len(names), md.num_rows, out, ctypes.byref(alloc.struct), ctypes.c_void_p(N.current_stream_handle()))
    N.check(status)  # the call has finished with `text` when it returns
    return [LogicalColumn.from_c(out[j], arrow_types[j], alloc) for j in range(len(names))], names


def parquet_read(files, *, columns=None, ignore_row_groups=None) -> LogicalTable:
    """Read Parquet files into a logical table.

    ``files``: a glob string, a path, or an iterable of paths; their tables
    are concatenated in order.  ``columns`` selects a subset of columns.
    ``ignore_row_groups`` only steers the reference's chunked multi-task read
    and is accepted for API compatibility."""
    from legate_dataframe.lib.csv import _concat

    paths = _file_list(files)
    if not paths:
        raise ValueError("no files to read")
    cols = None if columns is None else list(columns)
    try:
        parts, names = [], None
        for p in paths:
            part, names = _read_file_device(p, cols)
            parts.append(part)
        return LogicalTable(_concat(parts), names)
    except _NotOnDevice:
        pass
    tables = [pq.read_table(p, columns=cols) for p in paths]
    table = tables[0] if len(tables) == 1 else pa.concat_tables(tables)
    return LogicalTable.from_arrow(table)


def parquet_write(tbl: LogicalTable, path) -> None:
    """Write the table to ``path/part.0.parquet`` (the directory is created)."""
    out = pathlib.Path(path)
    out.mkdir(parents=True, exist_ok=True)
    pq.write_table(tbl.to_arrow(), out / "part.0.parquet")
