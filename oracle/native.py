"""The oracle's C part (``oracle/neumaier.c``): segment sums with Neumaier
compensation, the float SUM / MEAN checker of the full-size parity tests.

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.  ``build()`` compiles
it with gcc into ``oracle/liboracle_c.so`` (git-ignored, shipped with the
tree like the product library)."""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "neumaier.c"
LIB = HERE / "liboracle_c.so"
_lib = None


def build(force: bool = False) -> Path:
    if LIB.exists() and not force and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run(["gcc", "-O2", "-fno-fast-math", "-shared", "-fPIC", "-o", str(tmp), str(SRC), "-lm"],
                   check=True, capture_output=True, text=True)
    tmp.replace(LIB)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB))
        for name in ("ldf_oracle_segsum_f64", "ldf_oracle_segsum_f32"):
            f = getattr(L, name)
            f.restype = None
            f.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
        _lib = L
    return _lib


def segment_sums(x: np.ndarray, valid, offsets: np.ndarray):
    """(sums, valid counts) of the segments [offsets[s], offsets[s+1]) of x
    (float64 or float32, group-sorted), null rows skipped."""
    x = np.ascontiguousarray(x)
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    nseg = len(off) - 1
    out = np.empty(nseg, np.float64)
    cnt = np.empty(nseg, np.int64)
    v = None if valid is None else np.ascontiguousarray(valid, dtype=np.uint8)
    fn = lib().ldf_oracle_segsum_f64 if x.dtype == np.float64 else lib().ldf_oracle_segsum_f32
    assert x.dtype in (np.float64, np.float32)
    fn(x.ctypes.data, None if v is None else v.ctypes.data, off.ctypes.data, nseg, out.ctypes.data, cnt.ctypes.data)
    return out, cnt
