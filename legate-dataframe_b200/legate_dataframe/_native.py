"""ctypes binding of libldf_b200.so (the C ABI declared in include/ldf_b200.h).

Device memory for outputs and scratch is handed to the library through an
``ldf_allocator`` whose callbacks allocate torch CUDA tensors on the current
stream (the stand-in for legate's task memory resource); buffers the library
returns as outputs are adopted as tensors, scratch buffers are released back
to torch's caching allocator in stream order.

There is no CPU fallback: importing an op without the built library, or
calling it without a CUDA device, raises.
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

import torch

_LIB_PATH = Path(__file__).resolve().parent / "libldf_b200.so"

# ---- types (mirror include/ldf_b200.h) -----------------------------------
LDF_OK = 0
LDF_ERR_INVALID_ARGUMENT = 1
LDF_ERR_CUDA = 2
LDF_ERR_OUT_OF_MEMORY = 3
LDF_ERR_UNSUPPORTED = 4
LDF_ERR_TIMEOUT = 5
LDF_ERR_INTERNAL = 6

LDF_BOOL8 = 1
LDF_INT8 = 2
LDF_INT16 = 3
LDF_INT32 = 4
LDF_INT64 = 5
LDF_UINT8 = 6
LDF_UINT16 = 7
LDF_UINT32 = 8
LDF_UINT64 = 9
LDF_FLOAT32 = 10
LDF_FLOAT64 = 11
LDF_STRING = 12
LDF_TIMESTAMP_US = 13

TYPE_WIDTH = {
    LDF_BOOL8: 1, LDF_INT8: 1, LDF_UINT8: 1, LDF_INT16: 2, LDF_UINT16: 2,
    LDF_INT32: 4, LDF_UINT32: 4, LDF_FLOAT32: 4, LDF_INT64: 8, LDF_UINT64: 8,
    LDF_FLOAT64: 8, LDF_TIMESTAMP_US: 8, LDF_STRING: 16,
}

LDF_AGG = {
    "sum": 0, "min": 1, "max": 2, "count": 3, "count_all": 4, "mean": 5,
    "count_distinct": 6, "product": 7, "variance": 8, "stddev": 9,
}
NOALLOC_MAX_ROWS = 1 << 20  # LDF_B200_NOALLOC_MAX_ROWS

LDF_COUNT_ONLY_VALID = 0
LDF_COUNT_ONLY_NULL = 1
LDF_COUNT_ALL = 2


class ldf_column(ctypes.Structure):
    _fields_ = [
        ("type", ctypes.c_int32),
        ("nullable", ctypes.c_int32),
        ("size", ctypes.c_int64),
        ("data", ctypes.c_void_p),
        ("valid", ctypes.c_void_p),
        ("chars", ctypes.c_void_p),
        ("chars_base", ctypes.c_int64),
        ("num_chars", ctypes.c_int64),
    ]


ALLOC_FN = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)
DEALLOC_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)


class ldf_allocator(ctypes.Structure):
    _fields_ = [("ctx", ctypes.c_void_p), ("allocate", ALLOC_FN), ("deallocate", DEALLOC_FN)]


# Parquet page table (ldf_b200_parquet_decode)
LDF_PQ_DICT_PAGE, LDF_PQ_DATA_V1, LDF_PQ_DATA_V2 = 0, 1, 2
LDF_PQ_UNCOMPRESSED, LDF_PQ_SNAPPY = 0, 1
LDF_PQ_BOOLEAN, LDF_PQ_INT32, LDF_PQ_INT64, LDF_PQ_FLOAT, LDF_PQ_DOUBLE, LDF_PQ_BYTE_ARRAY = 0, 1, 2, 4, 5, 6


class ldf_parquet_page(ctypes.Structure):
    _fields_ = [("offset", ctypes.c_int64), ("compressed", ctypes.c_int64), ("uncompressed", ctypes.c_int64),
                ("row0", ctypes.c_int64), ("num_values", ctypes.c_int32), ("kind", ctypes.c_int32),
                ("encoding", ctypes.c_int32), ("codec", ctypes.c_int32), ("levels_bytes", ctypes.c_int32),
                ("dict", ctypes.c_int32), ("column", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class ldf_aggregation(ctypes.Structure):
    _fields_ = [
        ("in_col", ctypes.c_int32),
        ("kind", ctypes.c_int32),
        ("count_mode", ctypes.c_int32),
        ("out_type", ctypes.c_int32),
    ]


# ---- library ----------------------------------------------------------------
_lib = None
_lib_lock = threading.Lock()


def lib():
    """Load libldf_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lib_lock:
        if _lib is None:
            if not _LIB_PATH.exists():
                raise RuntimeError(
                    f"{_LIB_PATH} is missing: build it with "
                    "`python legate-dataframe_b200/build.py` (there is no CPU fallback)"
                )
            L = ctypes.CDLL(str(_LIB_PATH))
            P = ctypes.POINTER
            i32p = P(ctypes.c_int32)
            L.ldf_b200_join.argtypes = [
                P(ldf_column), ctypes.c_int32, P(ldf_column), ctypes.c_int32,
                i32p, i32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                i32p, ctypes.c_int32, i32p, ctypes.c_int32,
                P(ldf_column), P(ldf_allocator), ctypes.c_void_p,
            ]
            L.ldf_b200_groupby_aggregation.argtypes = [
                P(ldf_column), ctypes.c_int32, i32p, ctypes.c_int32,
                P(ldf_aggregation), ctypes.c_int32, P(ldf_column),
                P(ldf_allocator), ctypes.c_void_p,
            ]
            L.ldf_b200_sort.argtypes = [
                P(ldf_column), ctypes.c_int32, i32p, P(ctypes.c_uint8), ctypes.c_int32,
                ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, P(ldf_column),
                P(ldf_allocator), ctypes.c_void_p,
            ]
            L.ldf_b200_hash_partition.argtypes = [
                P(ldf_column), ctypes.c_int32, i32p, ctypes.c_int32, ctypes.c_int32,
                P(ldf_column), P(ctypes.c_int64), P(ldf_allocator), ctypes.c_void_p,
            ]
            L.ldf_b200_distinct.argtypes = [
                P(ldf_column), ctypes.c_int32, i32p, ctypes.c_int32, P(ldf_column),
                P(ldf_allocator), ctypes.c_void_p,
            ]
            L.ldf_b200_free_column.argtypes = [P(ldf_column), P(ldf_allocator), ctypes.c_void_p]
            L.ldf_b200_hash_partition_noalloc.argtypes = [
                P(ldf_column), ctypes.c_int32, i32p, ctypes.c_int32, ctypes.c_int32,
                P(ldf_column), P(ctypes.c_int64), ctypes.c_void_p,
            ]
            L.ldf_b200_hash_partition_noalloc.restype = ctypes.c_int
            L.ldf_b200_arrow_bits_to_bytes.argtypes = [
                ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
            ]
            L.ldf_b200_arrow_offsets_to_ranges.argtypes = [
                ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
            ]
            L.ldf_b200_test_stalled_lookback.argtypes = [ctypes.c_uint32, P(ldf_allocator), ctypes.c_void_p]
            L.ldf_b200_test_stalled_lookback.restype = ctypes.c_int
            L.ldf_b200_csv_read.argtypes = [
                ctypes.c_void_p, ctypes.c_int64, ctypes.c_char, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32,
                P(ldf_column), ctypes.POINTER(ctypes.c_int64), P(ldf_allocator), ctypes.c_void_p,
            ]
            L.ldf_b200_csv_read.restype = ctypes.c_int
            L.ldf_b200_parquet_decode.argtypes = [
                ctypes.c_void_p, ctypes.c_int64, P(ldf_parquet_page), ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, ctypes.c_int64,
                P(ldf_column), P(ldf_allocator), ctypes.c_void_p,
            ]
            L.ldf_b200_parquet_decode.restype = ctypes.c_int
            i64p = P(ctypes.c_int64)
            L.ldf_b200_parquet_pages.argtypes = [
                ctypes.c_void_p, ctypes.c_int64, i64p, i64p, i64p, i32p, i32p, i32p, ctypes.c_int32,
                P(ldf_parquet_page), ctypes.c_int32, i32p,
            ]
            L.ldf_b200_parquet_pages.restype = ctypes.c_int
            L.ldf_b200_arrow_bits_to_bytes.restype = ctypes.c_int
            L.ldf_b200_arrow_offsets_to_ranges.restype = ctypes.c_int
            L.ldf_b200_launch_count.restype = ctypes.c_ulonglong
            L.ldf_b200_profile_enable.argtypes = [ctypes.c_int]
            L.ldf_b200_profile_report.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int]
            L.ldf_b200_profile_report.restype = ctypes.c_int
            L.ldf_b200_last_error.restype = ctypes.c_char_p
            L.ldf_b200_version.restype = ctypes.c_char_p
            for name in ("ldf_b200_join", "ldf_b200_groupby_aggregation", "ldf_b200_sort",
                         "ldf_b200_hash_partition", "ldf_b200_distinct", "ldf_b200_free_column"):
                getattr(L, name).restype = ctypes.c_int
            _lib = L
    return _lib


def check(status: int) -> None:
    """Translate a C-ABI status into the exception type the reference raises
    (std::invalid_argument -> ValueError, runtime errors -> RuntimeError)."""
    if status == LDF_OK:
        return
    msg = lib().ldf_b200_last_error().decode("utf-8", "replace")
    if status in (LDF_ERR_INVALID_ARGUMENT, LDF_ERR_UNSUPPORTED):
        raise ValueError(msg)
    if status == LDF_ERR_OUT_OF_MEMORY:
        raise MemoryError(msg)
    raise RuntimeError(msg)


# ---- torch-backed allocator -------------------------------------------------
class TorchAllocator:
    """Allocate library buffers as torch uint8 CUDA tensors.

    Every live buffer is kept in ``self.live`` by address; outputs are
    ``adopt``-ed after the call, scratch is dropped by the deallocate callback.
    """

    def __init__(self, device: torch.device):
        self.device = device
        self.live: dict[int, torch.Tensor] = {}

        def _alloc(ctx, nbytes, stream):
            try:
                t = torch.empty(int(nbytes), dtype=torch.uint8, device=self.device)
            except Exception:  # noqa: BLE001 - report OOM as NULL
                return None
            p = t.data_ptr()
            self.live[p] = t
            return p

        def _free(ctx, ptr, nbytes, stream):
            self.live.pop(ptr, None)

        self._alloc_cb = ALLOC_FN(_alloc)
        self._free_cb = DEALLOC_FN(_free)
        self.struct = ldf_allocator(None, self._alloc_cb, self._free_cb)

    def adopt(self, ptr: int | None) -> torch.Tensor | None:
        if not ptr:
            return None
        return self.live.pop(ptr)


def current_stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("legate_dataframe (B200 build) needs a CUDA device; there is no CPU fallback")
    return torch.device("cuda", torch.cuda.current_device())


def int32_array(values) -> ctypes.Array:
    values = list(values)
    return (ctypes.c_int32 * max(len(values), 1))(*values)


def launch_count() -> int:
    """Kernels launched by libldf_b200.so so far in this process."""
    return int(lib().ldf_b200_launch_count())


def profile_enable(on: bool) -> None:
    """Bracket every library kernel launch with CUDA events on its stream."""
    lib().ldf_b200_profile_enable(1 if on else 0)


def profile_report(reset: bool = True) -> dict[str, tuple[int, float]]:
    """{kernel: (launches, total device ms)} collected while profiling."""
    n = lib().ldf_b200_profile_report(None, 0, 0)
    buf = ctypes.create_string_buffer(n + 1)
    lib().ldf_b200_profile_report(buf, n + 1, 1 if reset else 0)
    out = {}
    for line in buf.value.decode().splitlines():
        name, cnt, ms = line.split()
        out[name] = (int(cnt), float(ms))
    return out


def library_path() -> str:
    return os.fspath(_LIB_PATH)
