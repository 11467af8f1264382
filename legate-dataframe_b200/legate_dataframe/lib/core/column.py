"""LogicalColumn: one device-resident column in the legate physical layout.

Layout (mirrors legate-dataframe's PhysicalColumn, cpp/include/legate_dataframe/
core/column.hpp:454-671):
  * fixed width: ``data`` holds ``size`` values;
  * nullable columns carry a one-byte-per-row ``valid`` mask (1 = valid), the
    legate bool null mask, not an Arrow bitmask;
  * strings: ``data`` holds ``size`` inclusive global char ranges
    (legate ``Rect<1>``, two int64 each) into ``chars``; ``chars_base`` is the
    global position of ``chars[0]``.
A column is nullable iff its Arrow source had nulls (core/column.cpp:128).
"""

from __future__ import annotations

import ctypes
import warnings

import numpy as np
import pyarrow as pa
import torch

from legate_dataframe import _native as N

_FIXED = {
    pa.bool_(): N.LDF_BOOL8,
    pa.int8(): N.LDF_INT8,
    pa.int16(): N.LDF_INT16,
    pa.int32(): N.LDF_INT32,
    pa.int64(): N.LDF_INT64,
    pa.uint8(): N.LDF_UINT8,
    pa.uint16(): N.LDF_UINT16,
    pa.uint32(): N.LDF_UINT32,
    pa.uint64(): N.LDF_UINT64,
    pa.float32(): N.LDF_FLOAT32,
    pa.float64(): N.LDF_FLOAT64,
}
_NP_OF_LDF = {
    N.LDF_BOOL8: np.uint8, N.LDF_INT8: np.int8, N.LDF_INT16: np.int16, N.LDF_INT32: np.int32,
    N.LDF_INT64: np.int64, N.LDF_UINT8: np.uint8, N.LDF_UINT16: np.uint16, N.LDF_UINT32: np.uint32,
    N.LDF_UINT64: np.uint64, N.LDF_FLOAT32: np.float32, N.LDF_FLOAT64: np.float64,
    N.LDF_TIMESTAMP_US: np.int64,
}


def ldf_type_of(arrow_type: pa.DataType) -> int:
    if arrow_type in _FIXED:
        return _FIXED[arrow_type]
    if pa.types.is_string(arrow_type) or pa.types.is_large_string(arrow_type):
        return N.LDF_STRING
    if pa.types.is_timestamp(arrow_type) or pa.types.is_date64(arrow_type) or pa.types.is_duration(arrow_type):
        return N.LDF_TIMESTAMP_US
    if pa.types.is_date32(arrow_type):
        return N.LDF_INT32
    raise ValueError(f"unsupported Arrow type for the B200 path: {arrow_type}")


def _buffer_to_device(buf, start: int, nbytes: int, device) -> torch.Tensor:
    """Bytes [start, start + nbytes) of an Arrow buffer, copied to the device."""
    if buf is None or nbytes <= 0:
        return torch.empty(16, dtype=torch.uint8, device=device)
    host = np.frombuffer(buf, dtype=np.uint8, count=nbytes, offset=start)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")  # read-only view: torch only reads it
        return torch.from_numpy(host).to(device)


def _expand_bits(L, buf, bit_offset: int, n: int, device, stream) -> torch.Tensor:
    """One byte per row from an Arrow bitmap, expanded on the device."""
    out = torch.empty(max(n, 1), dtype=torch.uint8, device=device)
    if n:
        first = bit_offset >> 3
        nbytes = ((bit_offset & 7) + n + 7) >> 3
        bits = _buffer_to_device(buf, first, nbytes, device)
        N.check(L.ldf_b200_arrow_bits_to_bytes(bits.data_ptr(), bit_offset & 7, n, out.data_ptr(), stream))
    return out


class LogicalColumn:
    """A column resident in device memory (legate layout)."""

    def __init__(self, arrow_type, ldf_type, size, data, valid=None, chars=None, chars_base=0, num_chars=0):
        self.arrow_type = arrow_type
        self.ldf_type = ldf_type
        self.size = int(size)
        self.data = data
        self.valid = valid
        self.chars = chars
        self.chars_base = int(chars_base)
        self.num_chars = int(num_chars)

    # ---- construction -------------------------------------------------------
    @staticmethod
    def from_arrow(array, device=None) -> "LogicalColumn":
        """Copy an Arrow array to the device in the legate layout.  The Arrow
        buffers are copied as they are (values, the validity bitmap, string
        offsets and characters) and expanded on the device: the bitmap into
        one byte per row, the offsets into inclusive ranges (the library's
        ldf_b200_arrow_bits_to_bytes / ldf_b200_arrow_offsets_to_ranges)."""
        if isinstance(array, pa.ChunkedArray):
            array = array.combine_chunks()
        if device is None:
            device = N.require_cuda()
        t = ldf_type_of(array.type)
        n = len(array)
        if torch.device(device).type == "cpu":
            return LogicalColumn._from_arrow_host(array, t, n)
        off = array.offset
        bufs = array.buffers()
        L = N.lib()
        stream = torch.cuda.current_stream(device).cuda_stream
        valid = None
        if array.null_count > 0:
            valid = _expand_bits(L, bufs[0], off, n, device, stream)
        if t == N.LDF_STRING:
            ow = 8 if pa.types.is_large_string(array.type) else 4
            odt = np.int64 if ow == 8 else np.int32
            host_off = np.frombuffer(bufs[1], dtype=odt, count=n + 1, offset=off * ow) if n else np.zeros(1, odt)
            base, end = int(host_off[0]), int(host_off[-1])
            chars = _buffer_to_device(bufs[2], base, end - base, device)
            ranges = torch.empty(max(n, 1) * 16, dtype=torch.uint8, device=device)
            if n:
                d_off = _buffer_to_device(bufs[1], off * ow, (n + 1) * ow, device)
                N.check(L.ldf_b200_arrow_offsets_to_ranges(d_off.data_ptr(), ow, n, ranges.data_ptr(), stream))
            return LogicalColumn(array.type, t, n, ranges, valid, chars, base, end - base)
        if t == N.LDF_BOOL8:
            data = _expand_bits(L, bufs[1], off, n, device, stream)
        else:
            w = N.TYPE_WIDTH[t]
            data = _buffer_to_device(bufs[1], off * w, n * w, device)
        return LogicalColumn(array.type, t, n, data, valid)

    @staticmethod
    def _from_arrow_host(array, t: int, n: int) -> "LogicalColumn":
        """The same layout in host memory (numpy conversion on the host)."""
        def host(a: np.ndarray) -> torch.Tensor:
            a = np.ascontiguousarray(a)
            return torch.from_numpy(a.view(np.uint8).reshape(-1).copy())

        valid = host(np.asarray(array.is_valid(), dtype=np.uint8)) if array.null_count > 0 else None
        if t == N.LDF_STRING:
            large = pa.types.is_large_string(array.type)
            bufs = array.buffers()
            off = np.frombuffer(bufs[1], dtype=np.int64 if large else np.int32)[array.offset : array.offset + n + 1]
            off = off.astype(np.int64) if n else np.zeros(1, np.int64)
            base, end = int(off[0]), int(off[-1])
            chars = np.frombuffer(bufs[2], dtype=np.uint8)[base:end] if bufs[2] is not None else np.zeros(0, np.uint8)
            ranges = np.empty((n, 2), dtype=np.int64)
            ranges[:, 0] = off[:-1]
            ranges[:, 1] = off[1:] - 1
            return LogicalColumn(array.type, t, n, host(ranges), valid, host(chars), base, end - base)
        if t == N.LDF_BOOL8:
            vals = np.asarray(array.fill_null(False).to_numpy(zero_copy_only=False), dtype=np.uint8)
        else:
            storage = array if array.type in _FIXED else array.view(pa.int32() if t == N.LDF_INT32 else pa.int64())
            vals = np.asarray(storage.fill_null(0).to_numpy(zero_copy_only=False)).astype(_NP_OF_LDF[t], copy=False)
        return LogicalColumn(array.type, t, n, host(vals), valid)

    @staticmethod
    def from_torch(data: torch.Tensor, arrow_type, valid: torch.Tensor | None = None) -> "LogicalColumn":
        """Wrap an existing device tensor (fixed width) without copying."""
        t = ldf_type_of(arrow_type)
        raw = data.contiguous().view(torch.uint8).reshape(-1)
        v = None if valid is None else valid.contiguous().view(torch.uint8).reshape(-1)
        return LogicalColumn(arrow_type, t, data.numel(), raw, v)

    # ---- accessors ----------------------------------------------------------
    def nullable(self) -> bool:
        return self.valid is not None

    def num_rows(self) -> int:
        return self.size

    def dtype(self):
        return self.arrow_type

    def to_c(self) -> N.ldf_column:
        c = N.ldf_column()
        c.type = self.ldf_type
        c.nullable = 1 if self.valid is not None else 0
        c.size = self.size
        c.data = self.data.data_ptr() if self.data is not None else None
        c.valid = self.valid.data_ptr() if self.valid is not None else None
        c.chars = self.chars.data_ptr() if self.chars is not None else None
        c.chars_base = self.chars_base
        c.num_chars = self.num_chars
        return c

    @staticmethod
    def from_c(c: N.ldf_column, arrow_type, alloc: N.TorchAllocator) -> "LogicalColumn":
        """Adopt an output column produced by the library."""
        data = alloc.adopt(c.data)
        valid = alloc.adopt(c.valid) if c.nullable else None
        chars = alloc.adopt(c.chars) if c.type == N.LDF_STRING else None
        return LogicalColumn(arrow_type, c.type, c.size, data, valid, chars, c.chars_base, c.num_chars)

    # ---- back to the host -----------------------------------------------------
    def to_arrow(self) -> pa.Array:
        n = self.size
        w = N.TYPE_WIDTH[self.ldf_type]
        mask = None
        if self.valid is not None:
            mask = ~self.valid[:n].cpu().numpy().astype(bool)
        if self.ldf_type == N.LDF_STRING:
            ranges = self.data[: n * 16].cpu().numpy().view(np.int64).reshape(n, 2)
            chars = self.chars[: self.num_chars].cpu().numpy() if self.chars is not None else np.zeros(0, np.uint8)
            lo = ranges[:, 0] - self.chars_base
            ln = ranges[:, 1] - ranges[:, 0] + 1
            if mask is not None:
                ln = np.where(mask, 0, ln)
                lo = np.where(mask, 0, lo)
            offsets = np.zeros(n + 1, dtype=np.int64)
            np.cumsum(ln, out=offsets[1:])
            total = int(offsets[-1])
            if n and total:
                idx = np.repeat(lo - offsets[:-1], ln) + np.arange(total)
                packed = chars[idx]
            else:
                packed = np.zeros(0, np.uint8)
            large = total >= 2**31 or pa.types.is_large_string(self.arrow_type)
            typ = pa.large_string() if large else pa.string()
            off = offsets if large else offsets.astype(np.int32)
            validity = None
            if mask is not None:
                validity = pa.array(~mask).buffers()[1]
            arr = pa.Array.from_buffers(typ, n, [validity, pa.py_buffer(off), pa.py_buffer(packed)],
                                        null_count=int(mask.sum()) if mask is not None else 0)
            if not large and pa.types.is_large_string(self.arrow_type):
                arr = arr.cast(self.arrow_type)
            return arr
        vals = self.data[: n * w].cpu().numpy().view(_NP_OF_LDF[self.ldf_type])
        if self.ldf_type == N.LDF_BOOL8:
            arr = pa.array(vals.astype(bool), mask=mask, type=pa.bool_())
        elif self.arrow_type in _FIXED:
            arr = pa.array(vals, mask=mask, type=self.arrow_type)
        else:
            storage = pa.int32() if self.ldf_type == N.LDF_INT32 else pa.int64()
            arr = pa.array(vals, mask=mask, type=storage).view(self.arrow_type)
        return arr

    def __repr__(self) -> str:
        return f"LogicalColumn(type={self.arrow_type}, rows={self.size}, nullable={self.nullable()})"
