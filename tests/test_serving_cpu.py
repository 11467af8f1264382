"""Host logic of the batched/served path: device arena, memory-based
admission, request planning and the batch C-ABI argument checks.  CPU only."""

import ctypes
from collections import deque

import pytest
import torch

from legate_dataframe import _native as N
from legate_dataframe.serving import (GROUPBY, JOIN, DeviceArena, Request, _bind, admit, ldf_batch_request,
                                      ServerStats)


def test_request_struct_layout():
    # kind, vtype, n, m, k1, v1, k2, v2, vvalid, table, cap, o0..o3, out_cap
    assert ctypes.sizeof(ldf_batch_request) == 8 + 16 + 5 * 8 + 8 + 8 + 4 * 8 + 8


def test_arena_first_fit_and_coalescing():
    a = DeviceArena(1 << 20, device=None)
    offs = [a.alloc(1000) for _ in range(4)]
    assert offs == [0, 1024, 2048, 3072]
    a.release(offs[1], 1000)
    a.release(offs[2], 1000)
    assert a.alloc(2000) == 1024  # the two freed neighbours coalesced
    a.release(offs[0], 1000)
    a.release(1024, 2000)
    a.release(offs[3], 1000)
    assert a.free_bytes() == 1 << 20
    assert a._free == [(0, 1 << 20)]
    assert a.alloc((1 << 20) + 1) == -1


def _req(kind, n, ndv, dtype=torch.int64):
    k = torch.zeros(n, dtype=torch.int64)
    v = torch.zeros(n, dtype=dtype)
    if kind == JOIN:
        return Request(JOIN, k, v, k.clone(), v.clone(), ndv_hint=ndv)
    return Request(GROUPBY, k, v, ndv_hint=ndv)


def test_plan_sizes():
    g = _req(GROUPBY, 10_000, 1_000, torch.float64)
    total = g.plan(0.5)
    assert g.cap == 2001 and g.table_bytes == (g.cap + 1) * 8 * 8
    assert g.out_cap >= 1000 and g.out_bytes == g.out_cap * 24
    assert total == g.table_bytes + g.out_bytes
    j = _req(JOIN, 10_000, 1_000)
    j.plan(0.5)
    assert j.cap > j.m and j.table_bytes == j.cap * 16
    assert j.out_cap >= 10_000 * 10_000 // 1_000  # expected matches n*m/ndv
    assert j.out_bytes == j.out_cap * 32


def test_admission_is_fifo_and_memory_bounded():
    reqs = [_req(GROUPBY, 1000, 100) for _ in range(5)] + [_req(JOIN, 1_000_000, 100_000)] + \
           [_req(GROUPBY, 1000, 100) for _ in range(3)]
    for q in reqs:
        q.plan(0.5)
    small = reqs[0].table_bytes + reqs[0].out_bytes
    arena = DeviceArena(5 * (small + 512) + 4096, device=None)
    queue = deque(reqs)
    batch = admit(queue, arena, max_reqs=64, max_items=10_000, tile_rows=4096, load_factor=0.5)
    # the five small requests fit; the big join does not and nothing overtakes it
    assert len(batch) == 5 and queue[0].kind == JOIN and len(queue) == 4
    for q in batch:
        assert q.table_off >= 0 and q.out_off >= 0
    # nothing more fits while the batch holds its memory
    assert admit(queue, arena, 64, 10_000, 4096, 0.5) == []
    for q in batch:
        arena.release(q.table_off, q.table_bytes)
        arena.release(q.out_off, q.out_bytes)
    assert arena.free_bytes() == arena.nbytes


def test_admission_respects_request_and_item_capacity():
    reqs = deque(_req(GROUPBY, 5000, 100) for _ in range(10))
    arena = DeviceArena(1 << 30, device=None)
    assert len(admit(reqs, arena, max_reqs=4, max_items=10_000, tile_rows=1024, load_factor=0.5)) == 4
    # each request needs 2 table tiles + 5 row tiles + 2 = 9 items
    assert len(admit(reqs, arena, max_reqs=64, max_items=20, tile_rows=1024, load_factor=0.5)) == 2


def test_stats_summary():
    st = ServerStats(latencies_ms=[1.0] * 99 + [100.0], rows=1000, requests=100, batches=3, wall_s=2.0)
    s = st.summary()
    assert s["p50_ms"] == 1.0 and s["p99_ms"] > 1.0 and s["max_ms"] == 100.0
    assert s["req_per_s"] == 50.0 and s["rows_per_s"] == 500.0


def test_batch_abi_rejects_bad_arguments_without_gpu():
    L = _bind(N.lib())
    h = ctypes.c_void_p()
    st = L.ldf_b200_batch_create(0, 16, 4096, 1, None, ctypes.byref(h))
    assert st == N.LDF_ERR_INVALID_ARGUMENT
    assert b"bad engine config" in L.ldf_b200_last_error()
    st = L.ldf_b200_batch_run(None, None, 0)
    assert st == N.LDF_ERR_INVALID_ARGUMENT
    with pytest.raises(ValueError):
        N.check(st)
