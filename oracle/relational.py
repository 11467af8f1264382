"""numpy restatement of the reference's relational semantics (test oracle).

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.  Inputs and outputs
are ``pyarrow`` tables; row order of join / groupby results is unspecified
(tests compare after a canonical sort), sort results are exact.
"""

from __future__ import annotations

import math

import numpy as np
import pyarrow as pa

M64 = (1 << 64) - 1


# ---------------------------------------------------------------------------
# key factorization
# ---------------------------------------------------------------------------
def _values_and_valid(arr: pa.Array):
    arr = arr.combine_chunks() if isinstance(arr, pa.ChunkedArray) else arr
    valid = np.asarray(arr.is_valid(), dtype=bool)
    if pa.types.is_string(arr.type) or pa.types.is_large_string(arr.type):
        vals = np.array([v if v is not None else "" for v in arr.to_pylist()], dtype=object)
    elif pa.types.is_boolean(arr.type):
        vals = np.asarray(arr.fill_null(False).to_numpy(zero_copy_only=False), dtype=np.int64)
    elif pa.types.is_floating(arr.type):
        vals = np.asarray(arr.fill_null(0).to_numpy(zero_copy_only=False), dtype=np.float64)
        vals = np.where(vals == 0, 0.0, vals)  # -0.0 == 0.0
    else:
        storage = arr
        if pa.types.is_timestamp(arr.type) or pa.types.is_date(arr.type) or pa.types.is_duration(arr.type):
            storage = arr.view(pa.int64() if arr.type.bit_width == 64 else pa.int32())
        vals = np.asarray(storage.fill_null(0).to_numpy(zero_copy_only=False))
    return vals, valid


def _equality_values(arr: pa.Array):
    """Values under the equality of Arrow's hash kernels (grouper, hash join,
    hash_count_distinct): floats compare by their bit pattern, so 0.0 and -0.0
    are different keys and a NaN equals only a NaN with the same bits."""
    arr = arr.combine_chunks() if isinstance(arr, pa.ChunkedArray) else arr
    if pa.types.is_floating(arr.type):
        valid = np.asarray(arr.is_valid(), dtype=bool)
        v = np.asarray(arr.fill_null(0).to_numpy(zero_copy_only=False))
        return v.view({2: np.uint16, 4: np.uint32, 8: np.uint64}[v.dtype.itemsize]).astype(np.uint64), valid
    return _values_and_valid(arr)


def _codes(vals: np.ndarray) -> np.ndarray:
    """Dense codes of equal values (NaN == NaN)."""
    if len(vals) == 0:
        return np.zeros(0, dtype=np.int64)
    if vals.dtype == object:
        _, inv = np.unique(vals.astype(str), return_inverse=True)
    else:
        _, inv = np.unique(vals, return_inverse=True, equal_nan=True) if vals.dtype.kind == "f" else np.unique(
            vals, return_inverse=True
        )
    return inv.reshape(-1).astype(np.int64)


def _composite(code_cols: list[np.ndarray]) -> np.ndarray:
    if len(code_cols) == 1:
        return code_cols[0]
    m = np.stack(code_cols, axis=1)
    if len(m) == 0:
        return np.zeros(0, dtype=np.int64)
    _, inv = np.unique(m, axis=0, return_inverse=True)
    return inv.reshape(-1).astype(np.int64)


# ---------------------------------------------------------------------------
# join -- semantics of arrow_join_and_gather (cpp/src/join.cpp:168-228):
# nulls_equal: a null key equals a null key (process_key_column, join.cpp:117-162
# coalesces nulls and adds the validity as an extra key); otherwise rows with a
# null key never match.  LEFT/FULL unmatched rows get nulls on the other side
# (NULLIFY, cpp/src/join.cu:79-101); SEMI/ANTI keep lhs rows with/without match.
# ---------------------------------------------------------------------------
def join_indices(lhs: pa.Table, rhs: pa.Table, lhs_keys, rhs_keys, join_type: str, nulls_equal: bool):
    nl, nr = lhs.num_rows, rhs.num_rows
    lcodes, rcodes = [], []
    lbad = np.zeros(nl, dtype=bool)
    rbad = np.zeros(nr, dtype=bool)
    for lk, rk in zip(lhs_keys, rhs_keys):
        lv, lvalid = _equality_values(lhs.column(lk))
        rv, rvalid = _equality_values(rhs.column(rk))
        both = np.concatenate([lv, rv]) if len(lv) + len(rv) else lv
        codes = _codes(both)
        null_code = (codes.max() + 1) if len(codes) else 0
        codes = np.where(np.concatenate([lvalid, rvalid]), codes, null_code)
        lcodes.append(codes[:nl])
        rcodes.append(codes[nl:])
        if not nulls_equal:
            lbad |= ~lvalid
            rbad |= ~rvalid
    comp = _composite([np.concatenate([a, b]) for a, b in zip(lcodes, rcodes)])
    lc = np.where(lbad, -1, comp[:nl])
    rc = np.where(rbad, -2, comp[nl:])
    order = np.argsort(rc, kind="stable")
    rs = rc[order]
    lo = np.searchsorted(rs, lc, "left")
    hi = np.searchsorted(rs, lc, "right")
    cnt = np.where(lc >= 0, hi - lo, 0)
    if join_type == "semi":
        return np.nonzero(cnt > 0)[0], None
    if join_type == "anti":
        return np.nonzero(cnt == 0)[0], None
    total = int(cnt.sum())
    li = np.repeat(np.arange(nl), cnt)
    starts = np.repeat(lo - np.concatenate([[0], np.cumsum(cnt)[:-1]]), cnt)
    ri = order[starts + np.arange(total)] if total else np.zeros(0, dtype=np.int64)
    if join_type in ("left", "full"):
        um = np.nonzero(cnt == 0)[0]
        li = np.concatenate([li, um])
        ri = np.concatenate([ri, np.full(len(um), -1)])
    if join_type == "full":
        matched = np.zeros(nr, dtype=bool)
        matched[ri[ri >= 0]] = True
        ur = np.nonzero(~matched)[0]
        li = np.concatenate([li, np.full(len(ur), -1)])
        ri = np.concatenate([ri, ur])
    return li.astype(np.int64), ri.astype(np.int64)


def _take(col, idx: np.ndarray) -> pa.Array:
    col = col.combine_chunks() if isinstance(col, pa.ChunkedArray) else col
    mask = idx < 0
    ind = pa.array(np.where(mask, 0, idx), type=pa.int64(), mask=mask if mask.any() else None)
    if len(col) == 0:
        return pa.nulls(len(idx), type=col.type)
    return col.take(ind)


def join(lhs: pa.Table, rhs: pa.Table, lhs_keys, rhs_keys, join_type: str, nulls_equal: bool = True,
         lhs_out=None, rhs_out=None) -> pa.Table:
    lhs_out = list(lhs.column_names) if lhs_out is None else list(lhs_out)
    if rhs_out is None:
        rhs_out = [] if join_type in ("semi", "anti") else list(rhs.column_names)
    li, ri = join_indices(lhs, rhs, lhs_keys, rhs_keys, join_type, nulls_equal)
    cols = [_take(lhs.column(c), li) for c in lhs_out]
    if ri is not None:
        cols += [_take(rhs.column(c), ri) for c in rhs_out]
    return pa.Table.from_arrays(cols, names=lhs_out + (rhs_out if ri is not None else []))


# ---------------------------------------------------------------------------
# groupby -- semantics of the Acero hash_* aggregations
# (cpp/src/groupby_aggregation.cpp:41-94) and cudf's groupby with
# null_policy::INCLUDE (cpp/src/groupby_aggregation.cu:143): null keys form a
# group; SUM/MIN/MAX/MEAN skip nulls and are null without valid values; COUNT
# by CountOptions mode (.cu:33-44); COUNT_DISTINCT counts distinct valid
# values (+1 for null under mode "all").  Float SUM/MEAN use a Neumaier
# compensated sum per group.
# ---------------------------------------------------------------------------
def neumaier(xs) -> float:
    xs = list(xs)
    if not all(math.isfinite(x) for x in xs):
        # inf / NaN: IEEE propagation as in a plain sum (Arrow's sum of
        # [inf, 1.0] is inf; the compensation term would turn it into NaN)
        return float(sum(xs))
    s = 0.0
    c = 0.0
    for x in xs:
        t = s + x
        if abs(s) >= abs(x):
            c += (s - t) + x
        else:
            c += (x - t) + s
        s = t
    return s + c


def group_ids(table: pa.Table, keys):
    code_cols = []
    for k in keys:
        v, valid = _equality_values(table.column(k))
        c = _codes(v)
        null_code = (c.max() + 1) if len(c) else 0
        code_cols.append(np.where(valid, c, null_code))
    gid = _composite(code_cols)
    if len(gid) == 0:
        return gid, np.zeros(0, dtype=np.int64)
    # dense ids: a null row's placeholder value may be absent from the valid rows
    _, gid = np.unique(gid, return_inverse=True)
    gid = gid.reshape(-1).astype(np.int64)
    first = np.full(gid.max() + 1, len(gid), dtype=np.int64)
    np.minimum.at(first, gid, np.arange(len(gid)))
    return gid, first


def _count_mode(options) -> str:
    if options is None:
        return "only_valid"
    m = str(options).split("mode=")[-1].rstrip(")").strip().upper()
    return {"NULLS": "only_null", "ALL": "all"}.get(m, "only_valid")


def groupby(table: pa.Table, keys, aggs) -> pa.Table:
    """aggs: list of (in_col or None, kind or (kind, options), out_name)."""
    gid, first = group_ids(table, keys)
    G = len(first)
    out_cols = [table.column(k).combine_chunks().take(pa.array(first, type=pa.int64())) for k in keys]
    names = list(keys)
    order = np.argsort(gid, kind="stable")
    bounds = np.searchsorted(gid[order], np.arange(G + 1))
    for in_col, kind, out_name in aggs:
        options = None
        if isinstance(kind, tuple):
            kind, options = kind
        names.append(out_name)
        if kind == "count_all":
            out_cols.append(pa.array(np.bincount(gid, minlength=G).astype(np.int64)))
            continue
        arr = table.column(in_col).combine_chunks()
        vals, valid = _values_and_valid(arr)
        nvalid = np.bincount(gid[valid], minlength=G).astype(np.int64)
        nall = np.bincount(gid, minlength=G).astype(np.int64)
        if kind == "count":
            mode = _count_mode(options)
            v = {"only_valid": nvalid, "all": nall, "only_null": nall - nvalid}[mode]
            out_cols.append(pa.array(v, type=pa.int64()))
            continue
        if kind == "count_distinct":
            mode = _count_mode(options)
            codes = _codes(_equality_values(arr)[0])
            pairs = np.unique(np.stack([gid[valid], codes[valid]], axis=1), axis=0) if valid.any() else np.zeros((0, 2), np.int64)
            nd = np.bincount(pairs[:, 0], minlength=G).astype(np.int64) if len(pairs) else np.zeros(G, np.int64)
            has_null = (nall > nvalid).astype(np.int64)
            v = {"only_valid": nd, "all": nd + has_null, "only_null": has_null}[mode]
            out_cols.append(pa.array(v, type=pa.int64()))
            continue
        null_out = nvalid == 0
        t = arr.type
        if kind in ("sum", "mean"):
            if pa.types.is_floating(t):
                sums = np.zeros(G)
                sv = vals[order]
                vv = valid[order]
                for g in range(G):
                    seg = sv[bounds[g]:bounds[g + 1]][vv[bounds[g]:bounds[g + 1]]]
                    sums[g] = neumaier(seg.tolist())
                if kind == "mean":
                    with np.errstate(invalid="ignore", divide="ignore"):
                        res = sums / np.maximum(nvalid, 1)
                    out_cols.append(pa.array(res, mask=null_out, type=pa.float64()))
                else:
                    out_cols.append(pa.array(sums, mask=null_out, type=pa.float64()))
            else:
                unsigned = pa.types.is_unsigned_integer(t) or pa.types.is_boolean(t)
                acc = np.zeros(G, dtype=np.uint64 if unsigned else np.int64)
                np.add.at(acc, gid[valid], vals[valid].astype(acc.dtype))
                if kind == "mean":
                    res = acc.astype(np.float64) / np.maximum(nvalid, 1)
                    out_cols.append(pa.array(res, mask=null_out, type=pa.float64()))
                else:
                    out_cols.append(pa.array(acc, mask=null_out, type=pa.uint64() if unsigned else pa.int64()))
            continue
        if kind in ("min", "max"):
            if pa.types.is_floating(t):
                fill = np.inf if kind == "min" else -np.inf
                acc = np.full(G, fill)
                (np.fmin if kind == "min" else np.fmax).at(acc, gid[valid], vals[valid])
                res = pa.array(acc, mask=null_out, type=pa.float64()).cast(t)
            else:
                v = vals.astype(np.int64) if not pa.types.is_uint64(t) else vals.astype(np.uint64)
                info = np.iinfo(v.dtype)
                acc = np.full(G, info.max if kind == "min" else info.min, dtype=v.dtype)
                (np.minimum if kind == "min" else np.maximum).at(acc, gid[valid], v[valid])
                acc = np.where(null_out, 0, acc)
                storage = t
                if pa.types.is_timestamp(t) or pa.types.is_date(t):
                    storage = pa.int64() if t.bit_width == 64 else pa.int32()
                if pa.types.is_boolean(t):
                    res = pa.array(acc.astype(bool), mask=null_out, type=pa.bool_())
                else:
                    res = pa.array(acc.astype(storage.to_pandas_dtype()), mask=null_out, type=storage)
                    if storage != t:
                        res = res.view(t)
            out_cols.append(res)
            continue
        raise ValueError(f"oracle: unsupported aggregation {kind}")
    return pa.Table.from_arrays(out_cols, names=names)


# ---------------------------------------------------------------------------
# sort -- SortTask semantics (cpp/src/sort.cpp:312-376; the null-precedence
# flip of cpp/src/sort.cu:309-323 makes `nulls_at_end` hold for every key in
# either direction).  Within a key: values, then NaN, then null when
# nulls_at_end (reversed otherwise).  Stable (np.lexsort).
# ---------------------------------------------------------------------------
def sort_indices(table: pa.Table, keys, ascending=None, nulls_at_end=True) -> np.ndarray:
    ascending = [True] * len(keys) if ascending is None else list(ascending)
    lex = []  # least significant first for np.lexsort
    for k, asc in zip(keys, ascending):
        arr = table.column(k).combine_chunks()
        vals, valid = _values_and_valid(arr)
        nan = np.zeros(len(vals), dtype=bool)
        if vals.dtype.kind == "f":
            nan = np.isnan(vals) & valid
        cls = np.where(~valid, 2, np.where(nan, 1, 0))
        if not nulls_at_end:
            cls = 2 - cls
        ok = valid & ~nan
        rank = np.zeros(len(vals), dtype=np.int64)
        if ok.any():
            if vals.dtype == object:
                _, inv = np.unique(np.array([s.encode("utf-8") for s in vals[ok]], dtype=object), return_inverse=True)
            else:
                _, inv = np.unique(vals[ok], return_inverse=True)
            r = inv.reshape(-1).astype(np.int64)
            if not asc:
                r = r.max() - r
            rank[ok] = r
        lex.append((cls, rank))
    cols = []
    for cls, rank in reversed(lex):
        cols.append(rank)
        cols.append(cls)
    if not cols:
        return np.arange(table.num_rows)
    return np.lexsort(cols)


def sort(table: pa.Table, keys, ascending=None, nulls_at_end=True, limit=None) -> pa.Table:
    idx = sort_indices(table, keys, ascending, nulls_at_end)
    if limit is not None and abs(limit) < len(idx):
        idx = idx[limit:] if limit < 0 else idx[:limit]
    return table.take(pa.array(idx, type=pa.int64()))


# ---------------------------------------------------------------------------
# hash partition -- local step of task::repartition_by_hash
# (cpp/src/core/repartition_by_hash.cu:296-310): bucket = hash(keys) % nparts,
# rows grouped by bucket, input order within a bucket.  The hash is this
# project's (MurmurHash3 fmix64 mixing, restated from the kernels); the
# reference's cudf MURMUR3 bucket ids are unpinned by its tests.
# ---------------------------------------------------------------------------
def _mix64(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.uint64)
    with np.errstate(over="ignore"):
        x ^= x >> np.uint64(33)
        x *= np.uint64(0xFF51AFD7ED558CCD)
        x ^= x >> np.uint64(33)
        x *= np.uint64(0xC4CEB9FE1A85EC53)
        x ^= x >> np.uint64(33)
    return x


def _hash_combine(seed: np.ndarray, h: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        t = h + np.uint64(0x9E3779B97F4A7C15) + (seed << np.uint64(6)) + (seed >> np.uint64(2))
    return _mix64(seed ^ t)


def _hash_bytes(b: bytes) -> int:
    n = len(b)
    h = (0x27D4EB2F165667C5 ^ ((n * 0x9E3779B97F4A7C15) & M64)) & M64

    def mix(x):
        return int(_mix64(np.array([x], dtype=np.uint64))[0])

    i = 0
    while i + 8 <= n:
        w = int.from_bytes(b[i:i + 8], "little")
        h = (mix(h ^ w) + 0x165667B19E3779F9) & M64
        i += 8
    if i < n:
        w = int.from_bytes(b[i:], "little")
        h = (mix(h ^ w) + 0x165667B19E3779F9) & M64
    return mix(h)


def string_hashes(chars: np.ndarray, offsets: np.ndarray) -> np.ndarray:
    """`_hash_bytes` of every string [offsets[j], offsets[j+1]) of `chars`,
    vectorized over the strings: word w of all strings long enough to have it
    is folded in at once (the tail word zero-padded, as `_hash_bytes` does)."""
    chars = np.asarray(chars, dtype=np.uint8)
    off = np.asarray(offsets, dtype=np.int64)
    n = off[1:] - off[:-1]
    with np.errstate(over="ignore"):
        h = np.uint64(0x27D4EB2F165667C5) ^ (n.astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15))
    padded = np.concatenate([chars, np.zeros(8, np.uint8)])
    nwords = (n + 7) // 8
    for w in range(int(nwords.max()) if len(n) else 0):
        sel = np.nonzero(nwords > w)[0]
        start = off[:-1][sel] + 8 * w
        rem = np.minimum(n[sel] - 8 * w, 8)
        word = np.zeros(len(sel), np.uint64)
        for b in range(8):
            byte = padded[start + b].astype(np.uint64)
            byte = np.where(rem > b, byte, np.uint64(0))
            word |= byte << np.uint64(8 * b)
        with np.errstate(over="ignore"):
            h[sel] = _mix64(h[sel] ^ word) + np.uint64(0x165667B19E3779F9)
    return _mix64(h)


def _raw_bits(arr: pa.Array) -> tuple[np.ndarray, int]:
    t = arr.type
    width = t.bit_width // 8 if not pa.types.is_boolean(t) else 1
    if pa.types.is_boolean(t):
        raw = np.asarray(arr.fill_null(False).to_numpy(zero_copy_only=False), dtype=np.uint8).astype(np.uint64)
        return raw, 1
    storage = arr
    if not (pa.types.is_integer(t) or pa.types.is_floating(t)):
        storage = arr.view(pa.int64() if width == 8 else pa.int32())
    v = np.asarray(storage.fill_null(0).to_numpy(zero_copy_only=False))
    u = v.view({1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[width]).astype(np.uint64)
    return u, width


def row_hashes(table: pa.Table, keys) -> np.ndarray:
    n = table.num_rows
    h = np.full(n, 0x243F6A8885A308D3, dtype=np.uint64)
    for k in keys:
        arr = table.column(k).combine_chunks()
        valid = np.asarray(arr.is_valid(), dtype=bool)
        if pa.types.is_string(arr.type) or pa.types.is_large_string(arr.type):
            large = pa.types.is_large_string(arr.type)
            bufs = arr.buffers()
            offs = np.frombuffer(bufs[1], dtype=np.int64 if large else np.int32)[arr.offset:arr.offset + n + 1]
            chars = np.frombuffer(bufs[2], dtype=np.uint8) if bufs[2] is not None else np.zeros(0, np.uint8)
            hv = string_hashes(chars, offs.astype(np.int64)) if n else np.zeros(0, np.uint64)
        else:
            raw, width = _raw_bits(arr)
            with np.errstate(over="ignore"):
                hv = _mix64(raw + np.uint64((0x9E3779B97F4A7C15 * width) & M64))
        hv = np.where(valid, hv, np.uint64(0x5BD1E9955BD1E995))
        h = _hash_combine(h, hv)
    return h


def hash_partition(table: pa.Table, keys, nparts: int):
    h = row_hashes(table, keys)
    bucket = (h % np.uint64(nparts)).astype(np.int64)
    perm = np.argsort(bucket, kind="stable")
    counts = np.bincount(bucket, minlength=nparts)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    return table.take(pa.array(perm, type=pa.int64())), offsets.tolist(), bucket
