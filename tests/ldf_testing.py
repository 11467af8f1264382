"""Comparison helpers and golden-fixture access for the parity tests."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc

GOLDEN = Path(__file__).resolve().parent / "golden"


def load_golden():
    """Yield golden cases with their tables decoded."""
    man = json.loads((GOLDEN / "manifest.json").read_text())
    data = (GOLDEN / "golden.arrows").read_bytes()
    streams = man["streams"]

    def table(i):
        off, n = streams[i]
        return pa.ipc.open_stream(pa.py_buffer(data[off:off + n])).read_all()

    for case in man["cases"]:
        c = dict(case)
        c["tables"] = {k: table(v) for k, v in case["tables"].items()}
        yield c


def agg_spec(aggs_json):
    """Manifest aggregation list -> (in, kind or (kind, CountOptions), out)."""
    out = []
    for in_col, kind, name in aggs_json:
        if isinstance(kind, list):
            mode = {"ALL": "all", "NULLS": "only_null", "NON_NULL": "only_valid"}[kind[1]]
            kind = (kind[0], pc.CountOptions(mode=mode))
        out.append((in_col, kind, name))
    return out


def canonical(t: pa.Table, by=None) -> pa.Table:
    by = list(t.column_names) if by is None else list(by)
    if t.num_rows == 0 or not by:
        return t
    idx = pc.sort_indices(t, sort_keys=[(c, "ascending") for c in by], null_placement="at_start")
    return t.take(idx)


def _normalize_strings(t: pa.Table) -> pa.Table:
    cols = []
    for c in t.columns:
        if pa.types.is_large_string(c.type):
            c = c.cast(pa.string())
        cols.append(c.combine_chunks() if isinstance(c, pa.ChunkedArray) else c)
    return pa.Table.from_arrays(cols, names=t.column_names)


def assert_tables_equal(res: pa.Table, exp: pa.Table, sort_by="all", rtol: float = 0.0, check_types=True):
    """Exact equality (after a canonical sort) except float columns, which are
    compared with relative tolerance `rtol` (0 -> exact); validity must match."""
    assert res.column_names == exp.column_names, (res.column_names, exp.column_names)
    assert res.num_rows == exp.num_rows, (res.num_rows, exp.num_rows)
    res = _normalize_strings(res)
    exp = _normalize_strings(exp)
    if sort_by is not None:
        by = None if sort_by == "all" else sort_by
        res = canonical(res, by)
        exp = canonical(exp, by)
    for name in res.column_names:
        a = res.column(name).combine_chunks()
        b = exp.column(name).combine_chunks()
        if check_types:
            assert a.type == b.type, (name, a.type, b.type)
        va = np.asarray(a.is_valid())
        vb = np.asarray(b.is_valid())
        assert np.array_equal(va, vb), f"validity of {name} differs"
        if pa.types.is_floating(a.type):
            x = np.asarray(a.fill_null(0).to_numpy(zero_copy_only=False), dtype=np.float64)[va]
            y = np.asarray(b.fill_null(0).to_numpy(zero_copy_only=False), dtype=np.float64)[vb]
            both_nan = np.isnan(x) & np.isnan(y)
            if rtol == 0:
                ok = (x == y) | both_nan
            else:
                ok = (np.abs(x - y) <= rtol * np.maximum(np.abs(y), 1e-300)) | (x == y) | both_nan
            assert ok.all(), f"{name}: max rel err {np.max(np.abs(x - y) / np.maximum(np.abs(y), 1e-300))}"
        else:
            assert a.filter(pa.array(va)).equals(b.filter(pa.array(vb))), f"column {name} differs"


# Floats as keys or distinct values compare by bit pattern in Arrow's hash
# kernels: 0.0 != -0.0, and a NaN equals only a NaN with the same bits.
SPECIAL = np.array([0.0, -0.0, np.nan, -np.nan, 1.0, 0.0, -0.0, np.nan, 1.0, -np.nan], np.float64)


def special_float_tables(dtype=np.float64):
    """(groupby table, join lhs, join rhs) with 0.0/-0.0/NaN/-NaN keys."""
    x = SPECIAL.astype(dtype)
    t = pa.table({"k": x, "v": np.left_shift(1, np.arange(len(x), dtype=np.int64)), "w": x[::-1].copy()})
    lhs = pa.table({"k": x, "a": np.arange(len(x), dtype=np.int64)})
    rhs = pa.table({"k2": np.array([-0.0, np.nan, 2.0, 0.0, -np.nan, -0.0], dtype),
                    "b": np.arange(6, dtype=np.int64) + 100})
    return t, lhs, rhs
