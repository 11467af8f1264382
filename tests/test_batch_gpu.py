"""Batched execution (one graph replay for many joins/groupbys) and the
continuous-batching server: every batched result equals the oracle's result
for the request (the reference's CPU path: Acero hashjoin for joins; groupby
COUNT exact and SUM within 1e-12 of a Neumaier sum) and the per-op result of
the same request, alone and in a mix (bit-exact: integer columns, row sets
after a canonical sort, and float sums, which both paths compute from an exact
fixed-point sum); a 512-request slice of the served trace is checked request
by request; overflowing requests fall back to the per-op path."""

import numpy as np
import pyarrow as pa
import pytest
import torch

from ldf_testing import assert_tables_equal
from legate_dataframe import _native as N
from legate_dataframe.serving import (GROUPBY, JOIN, Autotuner, BatchEngine, DeviceArena, Request, Server,
                                      make_trace, read_result, run_one_op_per_launch, run_per_op)

pytestmark = pytest.mark.gpu

DEV = "cuda"
EMPTY_KEY = 0x7FF4DEAD7FF4BEEF  # the engine's empty-slot marker, as a key value


def _gen(seed):
    g = torch.Generator(device=DEV)
    g.manual_seed(seed)
    return g


def groupby_req(n, ndv, seed, dtype=torch.float64, null_frac=0.1, extra_keys=()):
    g = _gen(seed)
    k = torch.randint(0, max(ndv, 1), (n,), device=DEV, generator=g)
    for i, x in enumerate(extra_keys):
        if i < n:
            k[i] = x
    if dtype == torch.float64:
        v = torch.randn(n, dtype=torch.float64, device=DEV, generator=g)
    else:
        v = torch.randint(-(2**40), 2**40, (n,), device=DEV, generator=g)
    valid = torch.rand(n, device=DEV, generator=g) >= null_frac if null_frac else None
    return Request(GROUPBY, k, v, valid=valid, ndv_hint=ndv)


def join_req(n, m, ndv, seed):
    g = _gen(seed)
    k1 = torch.randint(0, max(ndv, 1), (n,), device=DEV, generator=g)
    v1 = torch.randint(-(2**40), 2**40, (n,), device=DEV, generator=g)
    k2 = torch.randint(0, max(ndv, 1), (m,), device=DEV, generator=g)
    v2 = torch.randint(-(2**40), 2**40, (m,), device=DEV, generator=g)
    return Request(JOIN, k1, v1, k2, v2, ndv_hint=ndv)


def per_op_arrow(q):
    t = run_per_op(q).to_arrow()
    if q.kind == GROUPBY:
        return t.rename_columns(["k", "sum", "count"])
    return t.rename_columns(["lk", "lv", "rk", "rv"])


def run_batch(reqs, arena_bytes=1 << 30, tile_rows=4096, ctas=2, lf=0.5):
    arena = DeviceArena(arena_bytes, torch.device(DEV))
    eng = BatchEngine(max_reqs=max(len(reqs), 1), max_items=1 << 16, tile_rows=tile_rows, ctas_per_sm=ctas)
    for q in reqs:
        q.plan(lf)
        q.table_off = arena.alloc(q.table_bytes)
        q.out_off = arena.alloc(q.out_bytes)
        assert q.table_off >= 0 and q.out_off >= 0
    eng.submit(reqs, arena)
    rows, ovf = eng.collect(len(reqs))
    out = []
    for q, r, o in zip(reqs, rows, ovf):
        q.rows_out = r
        out.append(None if o else read_result(q, arena))
    eng.close()
    return out, ovf


def oracle_arrow(q):
    """The request's result from the oracle: Acero hashjoin (the calls of
    JoinTask::cpu_variant) for joins; for groupbys the valid count per key
    and the sum of the valid values (Neumaier for float64, exact for int64)."""
    from oracle import arrow_ref as A
    from oracle import native

    k1 = q.k1.cpu().numpy()
    if q.kind == JOIN:
        lhs = pa.table({"lk": k1, "lv": q.v1.cpu().numpy()})
        rhs = pa.table({"rk": q.k2.cpu().numpy(), "rv": q.v2.cpu().numpy()})
        return A.join(lhs, rhs, ["lk"], ["rk"], "inner", True, use_threads=True)
    v = q.v1.cpu().numpy()
    ok = q.valid.cpu().numpy() if q.valid is not None else np.ones(len(k1), bool)
    order = np.argsort(k1, kind="stable")
    keys, start = np.unique(k1[order], return_index=True)
    off = np.append(start, len(k1)).astype(np.int64)
    if v.dtype == np.float64:
        sums, cnt = native.segment_sums(v[order], ok[order].astype(np.uint8), off)
    else:
        cnt = np.add.reduceat(ok[order].astype(np.int64), start) if len(k1) else np.zeros(0, np.int64)
        sums = np.add.reduceat(np.where(ok, v, 0)[order], start) if len(k1) else np.zeros(0, np.int64)
    return pa.table({"k": keys, "sum": pa.array(sums, mask=cnt == 0), "count": cnt})


def check(q, res, per_op=True):
    assert_tables_equal(res, oracle_arrow(q), check_types=False, rtol=1e-12)
    if per_op:
        assert_tables_equal(res, per_op_arrow(q), check_types=False)


@pytest.mark.parametrize("dtype", [torch.float64, torch.int64])
@pytest.mark.parametrize("n,ndv", [(1, 1), (1000, 100), (50_000, 5_000), (300_000, 300_000)])
def test_groupby_batch_matches_per_op(n, ndv, dtype):
    q = groupby_req(n, ndv, seed=n + ndv, dtype=dtype, extra_keys=(EMPTY_KEY, -1, 0))
    (res,), (ovf,) = run_batch([q])
    assert not ovf
    check(q, res)


@pytest.mark.parametrize("n,m,ndv", [(1, 1, 1), (1000, 800, 100), (50_000, 50_000, 5_000), (200_000, 30_000, 1_000),
                                     (0, 100, 10), (100, 0, 10)])
def test_join_batch_matches_per_op(n, m, ndv):
    q = join_req(n, m, ndv, seed=n * 3 + m)
    (res,), (ovf,) = run_batch([q])
    assert not ovf
    check(q, res)


def test_same_result_alone_and_in_the_mix():
    rng = np.random.default_rng(5)
    mix = []
    for i in range(96):
        n = int(np.clip(np.exp(np.log(20_000) + rng.standard_normal()), 100, 400_000))
        if i % 2:
            mix.append(join_req(n, n, max(1, n // 10), seed=1000 + i))
        else:
            mix.append(groupby_req(n, max(1, n // 10), seed=1000 + i))
    together, ovf = run_batch(mix, arena_bytes=6 << 30)
    assert not any(ovf)
    for i in (0, 1, 10, 31, 50, 95):
        q = mix[i]
        (alone,), (o,) = run_batch([q])
        assert not o
        # bit-identical, including float sums
        assert_tables_equal(together[i], alone, check_types=False)
        check(q, alone)


def test_overflow_is_flagged_and_server_falls_back():
    q = join_req(20_000, 20_000, 10, seed=3)  # ~40M output rows: far above the planned reservation
    q.ndv_hint = 20_000  # a wrong hint: the reservation is too small
    (_,), (ovf,) = run_batch([q])
    assert ovf
    g = groupby_req(5000, 50, seed=4, null_frac=0.0)
    g.v1[7] = 1e300  # outside the exact fixed-point range
    (_,), (ovf,) = run_batch([g])
    assert ovf
    srv = Server(arena_bytes=1 << 30, max_reqs=8, tile_rows=4096, ctas_per_sm=2, keep_results=True)
    q2 = join_req(20_000, 20_000, 100, seed=3)
    q2.ndv_hint = 20_000
    st = srv.serve([q2, g], realtime=False)
    srv.close()
    assert st.fallbacks == 2 and st.requests == 2
    assert_tables_equal(q2.result.rename_columns(["lk", "lv", "rk", "rv"]), per_op_arrow(q2), check_types=False)
    assert_tables_equal(g.result.rename_columns(["k", "sum", "count"]), per_op_arrow(g), check_types=False)


def test_server_results_match_per_op():
    reqs = make_trace(n_requests=48, rate=20_000.0, median_rows=5_000, max_rows=200_000, seed=9)
    srv = Server(arena_bytes=256 << 20, max_reqs=16, tile_rows=4096, ctas_per_sm=2, keep_results=True)
    st = srv.serve(reqs, realtime=True)
    srv.close()
    assert st.requests == 48 and st.batches >= 3  # small arena / slots: several batches, continuous admission
    for q in reqs:
        assert_tables_equal(q.result, per_op_arrow(q), check_types=False)
    base = run_one_op_per_launch(reqs[:8], realtime=False)
    assert base.requests == 8


def _np_mix(x):
    x = x.astype(np.uint64)
    with np.errstate(over="ignore"):
        x ^= x >> np.uint64(33)
        x *= np.uint64(0xFF51AFD7ED558CCD)
        x ^= x >> np.uint64(33)
        x *= np.uint64(0xC4CEB9FE1A85EC53)
        x ^= x >> np.uint64(33)
    return x


def _row_checksum(t: pa.Table) -> int:
    """Order-independent checksum of a table of int64 columns (row hashes of
    all columns together, summed modulo 2^64)."""
    h = np.zeros(t.num_rows, np.uint64)
    for j, c in enumerate(t.columns):
        x = c.combine_chunks().to_numpy().view(np.uint64) if t.num_rows else np.zeros(0, np.uint64)
        with np.errstate(over="ignore"):
            h = _np_mix(h + _np_mix(x + np.uint64(j + 1)))
    with np.errstate(over="ignore"):
        return int(h.sum(dtype=np.uint64))


def test_trace_slice_matches_oracle():
    """The first 512 requests of the served trace (LogNormal sizes, half
    joins, half groupbys), batched by the server and checked one by one:
    groupbys in full, joins by row count and an order-independent checksum of
    their rows (together about 2e8 output rows)."""
    reqs = make_trace(n_requests=512, seed=12)
    srv = Server(arena_bytes=16 << 30, tile_rows=16384, ctas_per_sm=8, load_factor=0.35, keep_results=True)
    served = 0
    for part in range(0, len(reqs), 64):  # 64 requests at a time keeps the host copies small
        chunk = reqs[part:part + 64]
        served += srv.serve(chunk, realtime=False).requests
        for q in chunk:
            exp = oracle_arrow(q)
            if q.kind == JOIN:
                got = q.result.rename_columns(["lk", "lv", "rk", "rv"])
                assert got.num_rows == exp.num_rows, q.rid
                assert _row_checksum(got) == _row_checksum(exp), q.rid
            else:
                assert_tables_equal(q.result.rename_columns(["k", "sum", "count"]), exp, check_types=False,
                                    rtol=1e-12)
            q.result = None
    srv.close()
    assert served == 512


def test_autotuner_persists_choice(tmp_path):
    calib = make_trace(n_requests=16, median_rows=2_000, max_rows=20_000, seed=2)
    tuner = Autotuner(cache_path=str(tmp_path / "tune.json"))
    cands = [(4096, 2, 0.5), (16384, 4, 0.35)]
    best = tuner.tune(calib, "unit", arena_bytes=256 << 20, candidates=cands)
    assert (best["tile_rows"], best["ctas_per_sm"], best["load_factor"]) in cands
    assert (tmp_path / "tune.json").exists()
    assert tuner.tune(calib, "unit", candidates=[(1, 1, 1.0)]) == best  # served from the cache


def test_engine_launches_are_counted():
    before = N.launch_count()
    q = groupby_req(1000, 10, seed=1)
    run_batch([q])
    assert N.launch_count() - before >= 4
