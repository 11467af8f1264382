"""The device Parquet decoder (ldf_b200_parquet_decode through
lib.parquet.parquet_read) against the reference's CPU reader, Arrow
(ParquetRead::cpu_variant, parquet.cpp): files Arrow wrote with Snappy or no
compression, dictionary or PLAIN encoding, data pages v1 and v2, nulls,
required columns, many row groups and pages, every supported type, a column
subset, several files, a chunk whose dictionary falls back to PLAIN, a
200 MB file; and files the device decoder does not take (gzip, nested)
still read through Arrow."""

import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq
import pytest

from ldf_testing import assert_tables_equal

pytestmark = pytest.mark.gpu


def device_read(paths, columns=None):
    from legate_dataframe.lib.parquet import parquet_read

    return parquet_read([str(p) for p in paths], columns=columns).to_arrow()


def table(n, seed, nulls=True):
    rng = np.random.default_rng(seed)
    m = (lambda p: rng.random(n) < p) if nulls else (lambda p: None)
    words = np.array([f"w{i}" * (i % 4 + 1) for i in range(3000)] + ["", "é€\U0001F642"], dtype=object)
    return pa.table({
        "b": pa.array(rng.random(n) < 0.3, mask=m(0.1)),
        "i8": pa.array(rng.integers(-128, 128, n), pa.int8(), mask=m(0.05)),
        "i16": pa.array(rng.integers(-2**15, 2**15, n), pa.int16()),
        "i32": pa.array(rng.integers(-2**31, 2**31, n), pa.int32(), mask=m(0.2)),
        "i64": pa.array(rng.integers(-2**63, 2**63 - 1, n), mask=m(0.1)),
        "lowcard": pa.array(rng.integers(0, 7, n), pa.int64(), mask=m(0.3)),
        "u8": pa.array(rng.integers(0, 256, n), pa.uint8()),
        "u16": pa.array(rng.integers(0, 2**16, n), pa.uint16(), mask=m(0.05)),
        "u32": pa.array(rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)),
        "u64": pa.array(rng.integers(0, 2**63, n, dtype=np.uint64) * 2 + 1, mask=m(0.05)),
        "f32": pa.array(rng.standard_normal(n).astype(np.float32), mask=m(0.05)),
        "f64": pa.array(rng.standard_normal(n), mask=m(0.1)),
        "s": pa.array(words[rng.integers(0, len(words), n)], mask=m(0.1)),
        "s_unique": pa.array([f"row{i}-{'x' * (i % 13)}" for i in range(n)]),
        "ts": pa.array(rng.integers(0, 10**15, n), pa.timestamp("us"), mask=m(0.05)),
        "d": pa.array(rng.integers(0, 20000, n).astype(np.int32), pa.date32()),
    })


@pytest.mark.parametrize("compression", ["snappy", "none"])
@pytest.mark.parametrize("dictionary", [True, False])
@pytest.mark.parametrize("version", ["1.0", "2.0"])
def test_parquet_matches_arrow(tmp_path, compression, dictionary, version):
    t = table(50_000, 1)
    p = tmp_path / "t.parquet"
    pq.write_table(t, p, compression=compression, use_dictionary=dictionary, data_page_version=version,
                   row_group_size=17_000, data_page_size=16 * 1024)
    assert_tables_equal(device_read([p]), pq.read_table(p), sort_by=None)


def test_parquet_subset_files_and_required(tmp_path):
    t = table(30_000, 2, nulls=False)
    schema = pa.schema([pa.field(f.name, f.type, nullable=False) for f in t.schema])
    paths = []
    for k in range(3):
        p = tmp_path / f"p{k}.parquet"
        pq.write_table(t.slice(k * 10_000, 10_000).cast(schema) if k != 1 else t.slice(k * 10_000, 10_000), p)
        paths.append(p)
    cols = ["s", "f64", "i8", "b"]
    exp = pa.concat_tables([pq.read_table(p, columns=cols) for p in paths], promote_options="permissive")
    assert_tables_equal(device_read(paths, cols), exp, sort_by=None)


def test_parquet_dictionary_fallback_and_long_runs(tmp_path):
    rng = np.random.default_rng(3)
    n = 200_000
    t = pa.table({"x": rng.standard_normal(n), "s": pa.array([f"{v:.12f}" for v in rng.standard_normal(n)]),
                  "c": pa.array(np.repeat(np.arange(5), n // 5), pa.int32()), "z": pa.array([None] * n, pa.int64())})
    p = tmp_path / "f.parquet"
    pq.write_table(t, p, dictionary_pagesize_limit=64 * 1024)
    assert_tables_equal(device_read([p]), pq.read_table(p), sort_by=None)


def test_parquet_200mb(tmp_path):
    rng = np.random.default_rng(4)
    n = 8_000_000
    t = pa.table({"k": rng.integers(0, 10**7, n), "x": rng.standard_normal(n),
                  "s": pa.array(np.char.mod("w%06d", rng.integers(0, 10**6, n)).astype(object)),
                  "i": pa.array(rng.integers(-1000, 1000, n), pa.int32(), mask=rng.random(n) < 0.02)})
    p = tmp_path / "big.parquet"
    pq.write_table(t, p)
    assert p.stat().st_size > 100e6
    assert_tables_equal(device_read([p]), pq.read_table(p), sort_by=None)


def test_parquet_not_on_device_reads_through_arrow(tmp_path):
    t = table(5_000, 5)
    p = tmp_path / "g.parquet"
    pq.write_table(t, p, compression="gzip")
    assert_tables_equal(device_read([p]), pq.read_table(p), sort_by=None)
    nested = pa.table({"l": pa.array([[1, 2], [3]], pa.list_(pa.int64())), "a": [1, 2]})
    q = tmp_path / "n.parquet"
    pq.write_table(nested, q)
    assert device_read([q], ["a"]).column("a").to_pylist() == [1, 2]


def _big_string_pages(tmp_path, compression, dictionary, version="1.0"):
    """A file whose byte-array pages are large enough for the chain path
    (dictionary pages of ~1 MB, PLAIN pages of ~1 MB) mixed with small ones."""
    rng = np.random.default_rng(8)
    n = 300_000
    words = np.array([f"k{i:07d}-" + "z" * (i % 11) for i in range(120_000)], dtype=object)
    t = pa.table({"s": pa.array(words[rng.integers(0, len(words), n)], mask=rng.random(n) < 0.05),
                  "run": pa.array(np.repeat(np.array(["aaaa" * 20, "b", ""], dtype=object), n // 3)),
                  "x": pa.array(rng.integers(0, 2**40, n))})
    p = tmp_path / f"big_{compression}_{dictionary}_{version}.parquet"
    pq.write_table(t, p, compression=compression, use_dictionary=dictionary, data_page_version=version,
                   row_group_size=150_000)
    return p


@pytest.mark.parametrize("compression", ["snappy", "none"])
@pytest.mark.parametrize("dictionary", [True, False])
@pytest.mark.parametrize("version", ["1.0", "2.0"])
def test_parquet_large_byte_array_pages(tmp_path, compression, dictionary, version):
    """Pages decoded by the whole GPU (Snappy element chains and dictionary
    length-prefix chains ranked in parallel) beside the per-page kernels."""
    p = _big_string_pages(tmp_path, compression, dictionary, version)
    assert_tables_equal(device_read([p]), pq.read_table(p), sort_by=None)


def _first_pages(path, column):
    """(payload offset, compressed bytes, kind, uncompressed bytes) of every page of a column."""
    from legate_dataframe.lib import parquet as P

    pf = pq.ParquetFile(path)
    _, idx, physical, _, _, _ = P._column_specs(pf, [column])
    data = np.fromfile(path, dtype=np.uint8)
    pages, n = P._page_table(data, pf.metadata, idx, physical)
    return data, [(pages[k].offset, pages[k].compressed, pages[k].kind, pages[k].uncompressed) for k in range(n)]


@pytest.mark.parametrize("which", ["chain_dictionary", "warp_data"])
def test_parquet_malformed_snappy_page_raises(tmp_path, which):
    """A Snappy stream whose first element copies from before the start is
    rejected with the page number, on both decoding paths."""
    p = _big_string_pages(tmp_path, "snappy", True)
    data, pages = _first_pages(p, "s")
    if which == "chain_dictionary":  # large enough for the chain path
        off, size, _, _ = next(pg for pg in pages if pg[2] == 0 and pg[3] >= 131072)
    else:  # small enough for the per-page kernel
        off, size, _, _ = next(pg for pg in pages if pg[2] != 0 and pg[3] < 131072)
    i = off
    while data[i] & 0x80:  # the length preamble
        i += 1
    data[i + 1] = 0x01  # a copy of 4 bytes at offset 0 * 256 + next byte, before any output
    data[i + 2] = 0x05
    q = tmp_path / "bad.parquet"
    data.tofile(q)
    with pytest.raises(ValueError, match="Parquet page"):
        device_read([q], ["s"])


def test_parquet_truncated_dictionary_raises(tmp_path):
    """An uncompressed dictionary page whose last length prefix runs past
    its data (the chain path for large dictionaries) is rejected."""
    p = _big_string_pages(tmp_path, "none", True)
    data, pages = _first_pages(p, "s")
    off, size, _, _ = next(pg for pg in pages if pg[2] == 0)
    assert size >= 16384
    x = off
    while x + 4 <= off + size:  # walk to the last entry
        ln = int(data[x]) | int(data[x + 1]) << 8 | int(data[x + 2]) << 16 | int(data[x + 3]) << 24
        if x + 4 + ln >= off + size:
            break
        x += 4 + ln
    data[x + 3] = 0x7F  # its length now runs far past the page
    q = tmp_path / "trunc.parquet"
    data.tofile(q)
    with pytest.raises(ValueError, match="Parquet page"):
        device_read([q], ["s"])
