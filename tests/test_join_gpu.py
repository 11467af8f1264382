"""Parity of the sm_100a hash join (through the C ABI) with the oracle and
the golden vectors: every join type, nulls_equal both ways, int/float/string
and multi-column keys, duplicates, empty tables, and the single-pass (unique
build keys) and two-pass (repeated build keys) probe paths."""

import zlib

import numpy as np
import pyarrow as pa
import pytest

from ldf_testing import assert_tables_equal, load_golden
from oracle import relational as R

pytestmark = pytest.mark.gpu

HOW = {"inner": 0, "left": 1, "full": 2, "semi": 3, "anti": 4}
JOIN_CASES = [c for c in load_golden() if c["op"] == "join"]


def run_join(lhs, rhs, lk, rk, how, nulls_equal=True, lo=None, ro=None):
    from legate_dataframe import LogicalTable
    from legate_dataframe.lib.join import JoinType, join

    res = join(LogicalTable.from_arrow(lhs), LogicalTable.from_arrow(rhs), lhs_keys=lk, rhs_keys=rk,
               join_type=JoinType(HOW[how]), lhs_out_columns=lo, rhs_out_columns=ro, nulls_equal=nulls_equal)
    return res.to_arrow()


@pytest.mark.parametrize("case", JOIN_CASES, ids=[c["name"] for c in JOIN_CASES])
def test_join_golden(case):
    t = case["tables"]
    res = run_join(t["lhs"], t["rhs"], case["lhs_keys"], case["rhs_keys"], case["how"], case["nulls_equal"],
                   case["lhs_out"], case["rhs_out"])
    assert_tables_equal(res, t["expected"], check_types=False)


def _keys(rng, n, kind, key_range, null_p):
    mask = rng.random(n) < null_p if null_p else None
    if kind == "string":
        v = [f"key-{x:05d}" * (1 + x % 3) for x in rng.integers(0, key_range, n)]
        if mask is not None:
            v = [None if m else s for s, m in zip(v, mask)]
        return pa.array(v, pa.string())
    if kind.startswith("float"):
        return pa.array(rng.integers(0, key_range, n).astype(kind), mask=mask)
    return pa.array(rng.integers(0, key_range, n).astype(kind), mask=mask)


@pytest.mark.parametrize("how", list(HOW))
@pytest.mark.parametrize("nulls_equal", [True, False])
@pytest.mark.parametrize("kind", ["int32", "int64", "float64", "string", "uint8"])
def test_join_random_parity(how, nulls_equal, kind):
    rng = np.random.default_rng(zlib.crc32(f"{how}{nulls_equal}{kind}".encode()))
    nl, nr = 3000, 2000
    kr = 200 if kind != "uint8" else 50
    lhs = pa.table({"lk": _keys(rng, nl, kind, kr, 0.05), "lp": pa.array(rng.normal(size=nl), mask=rng.random(nl) < .1),
                    "ls": pa.array([f"l{i}" for i in range(nl)])})
    rhs = pa.table({"rk": _keys(rng, nr, kind, kr, 0.05), "rp": rng.integers(-9, 9, nr).astype(np.int16),
                    "rb": pa.array(rng.random(nr) < 0.5)})
    res = run_join(lhs, rhs, ["lk"], ["rk"], how, nulls_equal)
    exp = R.join(lhs, rhs, ["lk"], ["rk"], how, nulls_equal)
    assert_tables_equal(res, exp)


@pytest.mark.parametrize("how", list(HOW))
def test_join_multikey(how):
    rng = np.random.default_rng(7)
    n = 4000
    lhs = pa.table({"a": _keys(rng, n, "int32", 20, 0.05), "b": _keys(rng, n, "string", 15, 0.05),
                    "v": np.arange(n)})
    rhs = pa.table({"c": _keys(rng, n // 2, "int32", 20, 0.05), "d": _keys(rng, n // 2, "string", 15, 0.05),
                    "w": np.arange(n // 2) * 3})
    for ne in (True, False):
        res = run_join(lhs, rhs, ["a", "b"], ["c", "d"], how, ne)
        exp = R.join(lhs, rhs, ["a", "b"], ["c", "d"], how, ne)
        assert_tables_equal(res, exp)


@pytest.mark.parametrize("how", ["inner", "left", "full"])
def test_join_unique_build_single_pass(how):
    # unique build keys take the one-pass probe with look-back offsets
    rng = np.random.default_rng(3)
    nb, npb = 300_000, 1_000_000
    bk = rng.permutation(nb).astype(np.int32)
    pk = np.where(rng.random(npb) < 0.8, rng.integers(0, nb, npb), rng.integers(nb, 2 * nb, npb)).astype(np.int32)
    rhs = pa.table({"k": bk, "p0": rng.integers(-2**40, 2**40, nb), "p1": rng.integers(-2**40, 2**40, nb)})
    lhs = pa.table({"k": pa.array(pk, mask=rng.random(npb) < 0.05), "x": rng.random(npb)})
    res = run_join(lhs, rhs, ["k"], ["k"], how, True, ["k", "x"], ["p0", "p1"])
    exp = R.join(lhs, rhs, ["k"], ["k"], how, True, ["k", "x"], ["p0", "p1"])
    assert_tables_equal(res, exp)


def test_join_1m_x_1m_uniform_int64_keys():
    # the reference benchmark shape: 1M x 1M int64 keys U[0, 2^20), seeds 1 and 2
    l_rng, r_rng = np.random.default_rng(1), np.random.default_rng(2)
    n = 1_000_000
    lhs = pa.table({"key": l_rng.integers(0, 1 << 20, n), "payload": l_rng.integers(-2**40, 2**40, n)})
    rhs = pa.table({"key_r": r_rng.integers(0, 1 << 20, n), "payload_r": r_rng.integers(-2**40, 2**40, n)})
    res = run_join(lhs, rhs, ["key"], ["key_r"], "inner")
    exp = R.join(lhs, rhs, ["key"], ["key_r"], "inner")
    assert res.num_rows == exp.num_rows
    assert_tables_equal(res, exp)


@pytest.mark.parametrize("how", list(HOW))
def test_join_empty(how):
    e = pa.table({"k": pa.array([], pa.int64()), "v": pa.array([], pa.float64())})
    f = pa.table({"k": pa.array([1, 2, 2], pa.int64()), "v": pa.array([1.0, 2.0, 3.0])})
    for lhs, rhs in ((e, f), (f, e), (e, e)):
        rhs = rhs.rename_columns(["kr", "w"])
        res = run_join(lhs, rhs, ["k"], ["kr"], how)
        exp = R.join(lhs, rhs, ["k"], ["kr"], how)
        assert_tables_equal(res, exp)


def test_join_all_null_keys():
    lhs = pa.table({"k": pa.array([None] * 5, pa.int32()), "v": np.arange(5)})
    rhs = pa.table({"kr": pa.array([None, 1, None], pa.int32()), "w": np.arange(3)})
    for how in HOW:
        for ne in (True, False):
            res = run_join(lhs, rhs, ["k"], ["kr"], how, ne)
            exp = R.join(lhs, rhs, ["k"], ["kr"], how, ne)
            assert_tables_equal(res, exp)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("how", ["inner", "left", "full", "semi", "anti"])
def test_join_special_float_keys_by_bits(how, dtype):
    from ldf_testing import special_float_tables

    _, lhs, rhs = special_float_tables(dtype)
    res = run_join(lhs, rhs, ["k"], ["k2"], how)
    exp = R.join(lhs, rhs, ["k"], ["k2"], how, True)
    assert_tables_equal(res, exp, sort_by=[c for c in exp.column_names if c in ("a", "b")], check_types=False)


@pytest.mark.parametrize("how", ["inner", "left", "full", "semi", "anti"])
@pytest.mark.parametrize("layout", ["fits", "fits_nullable", "too_wide"])
@pytest.mark.parametrize("dups", [False, True])
def test_join_mixed_width_outputs(how, layout, dups):
    # int32 keys with rhs output columns of every width (1, 2, 4, 8 bytes,
    # bool, float32), nullable or not, several int64 columns, duplicate and
    # null keys
    rng = np.random.default_rng(hash((how, layout, dups)) % 2**32)
    nb, nl = 3000, 5000
    bkeys = rng.integers(0, 2500 if dups else 10**6, nb).astype(np.int32)
    if not dups:
        bkeys = rng.permutation(np.arange(nb, dtype=np.int32) * 3)
    # "fits": no nulls; "fits_nullable": nullable key and int16; "too_wide": three int64 columns
    kmask = (rng.random(nb) < 0.03) if layout == "fits_nullable" else None
    rcols = {"rk": pa.array(bkeys, mask=kmask)}
    rcols["r8"] = pa.array(rng.integers(-100, 100, nb).astype(np.int8))
    rcols["r16"] = pa.array(rng.integers(-30000, 30000, nb).astype(np.int16),
                            mask=(rng.random(nb) < 0.2) if layout == "fits_nullable" else None)
    rcols["rb"] = pa.array(rng.random(nb) < 0.5)
    rcols["rf"] = pa.array(rng.normal(size=nb).astype(np.float32))
    if layout != "fits_nullable":
        rcols["r64"] = pa.array(rng.integers(-2**60, 2**60, nb))
    if layout == "too_wide":
        rcols["r64b"] = pa.array(rng.integers(-2**60, 2**60, nb))
        rcols["r64c"] = pa.array(rng.integers(-2**60, 2**60, nb))
    rhs = pa.table(rcols)
    lk = np.where(rng.random(nl) < 0.7, bkeys[rng.integers(0, nb, nl)], rng.integers(-10**6, 0, nl)).astype(np.int32)
    lhs = pa.table({"lk": pa.array(lk, mask=rng.random(nl) < 0.03), "lv": rng.normal(size=nl)})
    ro = [] if how in ("semi", "anti") else None
    res = run_join(lhs, rhs, ["lk"], ["rk"], how, True, None, ro)
    exp = R.join(lhs, rhs, ["lk"], ["rk"], how, True, None, ro)
    assert_tables_equal(res, exp, check_types=False)


def test_join_repeated_row_counts():
    # 2M unique int32 build keys, 4M probe rows (80% hits, 5% null keys):
    # FULL, INNER and LEFT row counts equal a reference count on every repeat
    import torch

    from legate_dataframe import LogicalColumn, LogicalTable
    from legate_dataframe.lib.join import JoinType, join

    dev = torch.device("cuda")
    g = torch.Generator(device=dev)
    g.manual_seed(11)
    nb, npr = 2_000_000, 4_000_000
    bkey = torch.randperm(nb, device=dev, generator=g).to(torch.int32)
    hit = torch.rand(npr, device=dev, generator=g) < 0.8
    pkey = torch.where(hit, bkey[torch.randint(0, nb, (npr,), device=dev, generator=g)],
                       torch.randint(nb, 2 * nb, (npr,), device=dev, generator=g, dtype=torch.int32))
    pvalid = torch.rand(npr, device=dev, generator=g) >= 0.05
    lt = LogicalTable([LogicalColumn.from_torch(pkey, pa.int32(), valid=pvalid)], ["lk"])
    rt = LogicalTable([LogicalColumn.from_torch(bkey, pa.int32()),
                       LogicalColumn.from_torch(torch.arange(nb, device=dev), pa.int64())], ["rk", "rv"])
    vk = pkey[pvalid]
    inner = int(torch.isin(vk, bkey).sum())
    unmatched = int((~torch.isin(bkey, vk)).sum())
    expect = {JoinType.INNER: inner, JoinType.LEFT: npr, JoinType.FULL: npr + unmatched}
    for _ in range(6):
        for jt, n in expect.items():
            assert join(lt, rt, lhs_keys=["lk"], rhs_keys=["rk"], join_type=jt).num_rows() == n, jt


@pytest.mark.parametrize("how", list(HOW))
@pytest.mark.parametrize("nulls_equal", [True, False])
@pytest.mark.parametrize("kind", ["int32", "int64", "float64", "uint8"])
@pytest.mark.parametrize("dup", [False, True])
def test_join_radix_partitioned(how, nulls_equal, kind, dup, monkeypatch):
    # the radix-partitioned path (forced on small inputs): 256 hash partitions
    # + a null-key partition on both sides, per-partition table regions
    monkeypatch.setenv("LDF_B200_JOIN_PARTITION", "1")
    rng = np.random.default_rng(zlib.crc32(f"p{how}{nulls_equal}{kind}{dup}".encode()))
    nl, nr = 20000, 6000
    kr = (3000 if dup else 10**6) if kind != "uint8" else 200
    lhs = pa.table({"lk": _keys(rng, nl, kind, kr, 0.05), "lp": pa.array(rng.normal(size=nl), mask=rng.random(nl) < .1),
                    "li": rng.integers(-9, 9, nl).astype(np.int32)})
    rk = _keys(rng, nr, kind, kr, 0.05)
    rhs = pa.table({"rk": rk, "rp": rng.integers(-9, 9, nr).astype(np.int16), "rb": pa.array(rng.random(nr) < 0.5),
                    "r8": rng.integers(-2**60, 2**60, nr)})
    ro = [] if how in ("semi", "anti") else None
    res = run_join(lhs, rhs, ["lk"], ["rk"], how, nulls_equal, None, ro)
    exp = R.join(lhs, rhs, ["lk"], ["rk"], how, nulls_equal, None, ro)
    assert_tables_equal(res, exp)


@pytest.mark.parametrize("how", list(HOW))
def test_join_radix_partitioned_edges(how, monkeypatch):
    monkeypatch.setenv("LDF_B200_JOIN_PARTITION", "1")
    e = pa.table({"k": pa.array([], pa.int64()), "v": pa.array([], pa.float64())})
    f = pa.table({"k": pa.array([1, 2, 2], pa.int64()), "v": pa.array([1.0, 2.0, 3.0])})
    for lhs, rhs in ((e, f), (f, e), (e, e), (f, f)):
        rhs = rhs.rename_columns(["kr", "w"])
        assert_tables_equal(run_join(lhs, rhs, ["k"], ["kr"], how), R.join(lhs, rhs, ["k"], ["kr"], how))
    lhs = pa.table({"k": pa.array([None] * 5, pa.int32()), "v": np.arange(5)})
    rhs = pa.table({"kr": pa.array([None, 1, None], pa.int32()), "w": np.arange(3)})
    for ne in (True, False):
        assert_tables_equal(run_join(lhs, rhs, ["k"], ["kr"], how, ne), R.join(lhs, rhs, ["k"], ["kr"], how, ne))


@pytest.mark.parametrize("how", ["inner", "left", "full", "semi", "anti"])
@pytest.mark.parametrize("case", ["dense_perm", "dense_gaps", "dense_dup", "dense_nulls", "dense_two_nulls",
                                  "int64_edges", "uint64_high", "int8_negative"])
def test_join_dense_integer_keys(how, case):
    """Build keys whose value range is at most twice the build rows take a
    direct-address table (a repeated key falls back to the hash table).  Probe
    keys outside the range, at the int64 extremes (where a subtraction would
    wrap around), nulls on either side, and unsigned keys above 2^63."""
    rng = np.random.default_rng(zlib.crc32(f"{how}{case}".encode()))
    nb, nl = 5000, 12000
    i64 = np.iinfo(np.int64)
    if case == "dense_perm":
        bk = pa.array(rng.permutation(nb) - 1000)
        lk = pa.array(rng.integers(-3000, 6000, nl))
    elif case == "dense_gaps":
        bk = pa.array(rng.choice(2 * nb - 10, nb, replace=False) + 7)
        lk = pa.array(rng.integers(0, 2 * nb + 20, nl))
    elif case == "dense_dup":
        bk = pa.array(np.concatenate([np.arange(nb - 1), [17]]))
        lk = pa.array(rng.integers(-5, nb + 5, nl))
    elif case in ("dense_nulls", "dense_two_nulls"):
        m = np.zeros(nb, bool)
        m[[3] if case == "dense_nulls" else [3, 4000]] = True
        bk = pa.array(rng.permutation(nb), mask=m)
        lk = pa.array(rng.integers(0, nb + 100, nl), mask=rng.random(nl) < 0.1)
    elif case == "int64_edges":
        bk = pa.array(i64.max - rng.permutation(nb))
        lk = pa.array(np.concatenate([i64.min + rng.integers(0, 3 * nb, nl // 2),
                                      i64.max - rng.integers(0, 2 * nb, nl - nl // 2)]))
    elif case == "uint64_high":
        bk = pa.array((np.uint64(2**63) + rng.permutation(nb).astype(np.uint64)))
        lk = pa.array((np.uint64(2**63) + rng.integers(0, 2 * nb, nl).astype(np.uint64)))
    else:  # int8_negative: every value of int8, twice (a repeat: hash table)
        bk = pa.array(np.tile(np.arange(-128, 128, dtype=np.int8), 2))
        lk = pa.array(rng.integers(-128, 128, nl).astype(np.int8))
    rhs = pa.table({"rk": bk, "rv": np.arange(len(bk), dtype=np.int64), "rw": rng.normal(size=len(bk))})
    lhs = pa.table({"lk": lk, "lv": np.arange(len(lk), dtype=np.int32)})
    ro = None if how in ("semi", "anti") else ["rk", "rv", "rw"]
    for nulls_equal in (True, False):
        res = run_join(lhs, rhs, ["lk"], ["rk"], how, nulls_equal, ro=ro)
        exp = R.join(lhs, rhs, ["lk"], ["rk"], how, nulls_equal, rhs_out=ro)
        assert_tables_equal(res, exp)
