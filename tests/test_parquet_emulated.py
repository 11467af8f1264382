"""The device Parquet decoder's kernels run on the CPU against the oracle.

The Snappy decoder, the RLE / bit-packed hybrid cutter, the dictionary entry
table and the data-page kernel of legate-dataframe_b200/csrc/parquet.cu are
compiled as host C++ with tests/host_emulation/parquet_emu.cpp (one thread
per block, tiles of 8 rows, 48-byte Snappy input stages, a 256-byte output
ring, 64-byte Snappy batches and 32-byte dictionary stages, so every tile
boundary, run split, restage, chain through a batch and ring miss is
exercised) under AddressSanitizer.  The page table comes from the library's
own footer and page-header reader (lib/parquet.py); every column's values
and nulls are compared with the reference's CPU reader, Arrow
(ParquetRead::cpu_variant, parquet.cpp), on files Arrow wrote with Snappy or
no compression, dictionary or PLAIN encoding, data pages v1 and v2, nulls,
many pages and row groups, and every supported type.  The GPU launch
geometry is checked by tests/test_parquet_gpu.py."""

import math
import shutil
import struct
import subprocess
from pathlib import Path

import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq
import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "legate-dataframe_b200" / "csrc" / "parquet.cu"
EMU = ROOT / "tests" / "host_emulation" / "parquet_emu.cpp"

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")


def _section() -> str:
    src = SRC.read_text()
    sec = src[src.index("constexpr int kLanes"):src.index("unsigned pq_blocks(")]
    for a, b in (("constexpr int kLanes     = 32;", "constexpr int kLanes     = 1;"),
                 ("constexpr int kPqThreads = 128;", "constexpr int kPqThreads = 1;"),
                 ("constexpr int kPqTile    = 1024;", "constexpr int kPqTile    = 8;"),
                 # small stages and ring: restaging, long literals and far back-references are frequent
                 ("constexpr int kSnapIn    = 2048;", "constexpr int kSnapIn    = 48;"),
                 ("constexpr int kSnapWin   = 32768;", "constexpr int kSnapWin   = 256;"),
                 ("constexpr int kSnapBatchBytes = 1024;", "constexpr int kSnapBatchBytes = 64;"),
                 ("constexpr int kSnapShort      = 64;", "constexpr int kSnapShort      = 16;"),
                 ("constexpr int kDictStage = 8192;", "constexpr int kDictStage = 32;"),
                 # most byte-array pages through the chain path, four elements between checkpoints
                 ("constexpr int64_t kChainMinBytes = 131072;", "constexpr int64_t kChainMinBytes = 200;"),
                 ("constexpr int64_t kDictChainMinBytes = 16384;", "constexpr int64_t kDictChainMinBytes = 100;"),
                 ("constexpr int kChainLog          = 8;", "constexpr int kChainLog          = 2;")):
        assert a in sec, a
        sec = sec.replace(a, b)
    return sec


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    d = tmp_path_factory.mktemp("pq_emu")
    (d / "parquet_sections.inc").write_text(_section())
    exe = d / "pq_emu"
    cmd = ["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
           f"-I{ROOT / 'include'}", f"-I{d}", str(EMU), "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return exe


def decode(exe, path, tmp_path, columns=None):
    import sys

    sys.path.insert(0, str(ROOT / "legate-dataframe_b200"))
    from legate_dataframe.lib import parquet as P

    pf = pq.ParquetFile(path)
    md, asch = pf.metadata, pf.schema_arrow
    names, idx, physical, types, nullable, _ = P._column_specs(pf, columns)
    spec = [v for triple in zip(physical, types, nullable) for v in triple]
    data = np.fromfile(path, dtype=np.uint8)
    pages, npages = P._page_table(data, md, idx, spec[0::3])
    blob = struct.pack("<4q", len(data), npages, len(idx), md.num_rows) + data.tobytes()
    blob += bytes(memoryview(pages))[: npages * 64] + struct.pack(f"<{len(spec)}i", *spec)
    inp = tmp_path / "emu.bin"
    inp.write_bytes(blob)
    r = subprocess.run([str(exe), str(inp)], capture_output=True)
    assert r.returncode == 0, r.stderr.decode()[-3000:]
    lines = r.stdout.decode().splitlines()
    assert not lines[0].startswith("error"), lines[0]
    rows = int(lines[0].split()[1])
    out, k = {}, 1
    for n, i in zip(names, idx):
        t = asch.field(i).type
        vals = []
        for line in lines[k:k + rows]:
            assert line != "BADMASK"
            if line == "N":
                vals.append(None)
            elif line.startswith("S "):
                vals.append(bytes.fromhex(line[2:]).decode())
            elif line.startswith("F "):
                bits = int(line[2:], 16)
                vals.append(struct.unpack("<f", struct.pack("<I", bits & 0xFFFFFFFF))[0] if t == pa.float32()
                            else struct.unpack("<d", struct.pack("<Q", bits))[0])
            else:
                vals.append(int(line[2:]))
        out[n] = vals
        k += rows
    return out


def expected(path, columns=None):
    t = pq.read_table(path, columns=columns)
    out = {}
    for n in t.column_names:
        c = t.column(n)
        if pa.types.is_timestamp(c.type) or pa.types.is_date32(c.type):
            c = c.cast(pa.int64() if pa.types.is_timestamp(c.type) else pa.int32())
        out[n] = [int(v) if isinstance(v, bool) else v for v in c.to_pylist()]
    return out


def same(got, exp):
    assert got.keys() == exp.keys()
    for n in got:
        a, b = got[n], exp[n]
        assert len(a) == len(b), n
        for i, (u, v) in enumerate(zip(a, b)):
            if isinstance(v, float):
                assert u is not None and (math.isnan(u) and math.isnan(v) or struct.pack("<d", u) == struct.pack("<d", v)), (n, i, u, v)
            else:
                assert u == v, (n, i, u, v)


def table(n, seed, nulls=True):
    rng = np.random.default_rng(seed)
    m = (lambda p: rng.random(n) < p) if nulls else (lambda p: None)
    words = np.array([f"w{i}" * (i % 4 + 1) for i in range(300)] + ["", "é€\U0001F642"], dtype=object)
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
        "f64": pa.array(np.round(rng.standard_normal(n), int(rng.integers(0, 3))), mask=m(0.1)),
        "s": pa.array(words[rng.integers(0, len(words), n)], mask=m(0.1)),
        "s_unique": pa.array([f"row{i}-{'x' * (i % 13)}" for i in range(n)]),
        "ts": pa.array(rng.integers(0, 10**15, n), pa.timestamp("us"), mask=m(0.05)),
        "d": pa.array(rng.integers(0, 20000, n).astype(np.int32), pa.date32()),
    })


@pytest.mark.parametrize("compression", ["snappy", "none"])
@pytest.mark.parametrize("dictionary", [True, False])
@pytest.mark.parametrize("version", ["1.0", "2.0"])
def test_decode_matches_arrow(emu, tmp_path, compression, dictionary, version):
    t = table(3000, 1)
    path = tmp_path / "t.parquet"
    pq.write_table(t, path, compression=compression, use_dictionary=dictionary, data_page_version=version,
                   row_group_size=1100, data_page_size=2048)
    same(decode(emu, path, tmp_path), expected(path))


def test_required_columns_and_selection(emu, tmp_path):
    t = table(2000, 2, nulls=False)
    schema = pa.schema([pa.field(f.name, f.type, nullable=False) for f in t.schema])
    path = tmp_path / "r.parquet"
    pq.write_table(t.cast(schema), path, data_page_size=1024)
    same(decode(emu, path, tmp_path), expected(path))
    cols = ["s", "i64", "b"]
    same(decode(emu, path, tmp_path, cols), expected(path, cols))


def test_dictionary_fallback_to_plain_within_a_chunk(emu, tmp_path):
    """A dictionary that outgrows its page limit: the chunk's first pages
    are dictionary-encoded, the later ones PLAIN."""
    rng = np.random.default_rng(3)
    n = 40_000
    t = pa.table({"x": rng.standard_normal(n), "s": pa.array([f"{v:.12f}" for v in rng.standard_normal(n)])})
    path = tmp_path / "f.parquet"
    pq.write_table(t, path, dictionary_pagesize_limit=16 * 1024, data_page_size=8 * 1024)
    encs = pq.ParquetFile(path).metadata.row_group(0).column(0).encodings
    assert "PLAIN" in encs and "RLE_DICTIONARY" in encs
    same(decode(emu, path, tmp_path), expected(path))


def test_long_runs_and_all_null_pages(emu, tmp_path):
    n = 50_000
    t = pa.table({"c": pa.array(np.repeat(np.arange(5), n // 5), pa.int32()),
                  "z": pa.array([None] * n, pa.int64()),
                  "h": pa.array(np.where(np.arange(n) % 1000 == 0, None, 7), pa.int64())})
    path = tmp_path / "l.parquet"
    pq.write_table(t, path, data_page_size=4096)
    same(decode(emu, path, tmp_path), expected(path))


def test_page_walk_rejects_what_the_decoder_lacks(tmp_path):
    """ldf_b200_parquet_pages (the host page-header walk) refuses pages in
    other encodings, which sends parquet_read to Arrow, and reports headers
    cut short by the file's end as invalid input."""
    import sys

    sys.path.insert(0, str(ROOT / "legate-dataframe_b200"))
    from legate_dataframe.lib import parquet as P

    t = pa.table({"x": pa.array(np.arange(5000), pa.int64())})
    path = tmp_path / "delta.parquet"
    pq.write_table(t, path, use_dictionary=False, column_encoding={"x": "DELTA_BINARY_PACKED"})
    pf = pq.ParquetFile(path)
    _, idx, physical, _, _, _ = P._column_specs(pf, None)
    data = np.fromfile(path, dtype=np.uint8)
    with pytest.raises(P._NotOnDevice, match="encoding"):
        P._page_table(data, pf.metadata, idx, physical)

    path = tmp_path / "plain.parquet"
    pq.write_table(t, path, use_dictionary=False, data_page_size=1024)
    pf = pq.ParquetFile(path)
    data = np.fromfile(path, dtype=np.uint8)
    pages, n = P._page_table(data, pf.metadata, idx, physical)
    assert n > 1 and sum(pages[k].num_values for k in range(n)) == 5000
    cut = data[: pages[1].offset - 3]  # the second page's header runs past the end
    with pytest.raises(ValueError):
        P._page_table(cut, pf.metadata, idx, physical)


def test_snappy_overlapping_and_far_copies(emu, tmp_path):
    """PLAIN pages that Snappy turns into overlapping back-references (runs
    of one value, short periodic strings) and references further back than
    the output ring, mixed with literals of every length class."""
    rng = np.random.default_rng(5)
    n = 30_000
    period = np.array(["ab" * (i % 5 + 1) for i in range(n)], dtype=object)
    far = rng.integers(0, 2**62, 64)  # a block of values repeated every 512 bytes
    t = pa.table({"zeros": pa.array(np.zeros(n, np.int64)),
                  "runs": pa.array(np.repeat(rng.integers(0, 2**40, n // 100), 100)),
                  "period": pa.array(period),
                  "far": pa.array(np.tile(far, n // 64 + 1)[:n]),
                  "noise": pa.array(rng.integers(0, 2**63, n)),
                  "mixed": pa.array(np.where(rng.random(n) < 0.5, 7, rng.integers(0, 2**31, n)))})
    path = tmp_path / "s.parquet"
    pq.write_table(t, path, use_dictionary=False, compression="snappy", data_page_size=64 * 1024)
    same(decode(emu, path, tmp_path), expected(path))


def _emu_run(exe, path, tmp_path, columns=None):
    import sys

    sys.path.insert(0, str(ROOT / "legate-dataframe_b200"))
    from legate_dataframe.lib import parquet as P

    pf = pq.ParquetFile(path)
    names, idx, physical, types, nullable, _ = P._column_specs(pf, columns)
    spec = [v for triple in zip(physical, types, nullable) for v in triple]
    data = np.fromfile(path, dtype=np.uint8)
    pages, npages = P._page_table(data, pf.metadata, idx, spec[0::3])
    blob = struct.pack("<4q", len(data), npages, len(idx), pf.metadata.num_rows) + data.tobytes()
    blob += bytes(memoryview(pages))[: npages * 64] + struct.pack(f"<{len(spec)}i", *spec)
    inp = tmp_path / "emu_bad.bin"
    inp.write_bytes(blob)
    r = subprocess.run([str(exe), str(inp)], capture_output=True)
    assert r.returncode == 0, r.stderr.decode()[-3000:]
    return r.stdout.decode().splitlines()[0], [(pages[k].offset, pages[k].uncompressed, pages[k].kind)
                                              for k in range(npages)]


@pytest.mark.parametrize("target", ["chain", "warp"])
def test_malformed_snappy_page_is_reported(emu, tmp_path, target):
    """A first element that copies from before the stream's start makes the
    decode fail with that page's number, through the chain kernels (pages
    from 200 bytes here) and through the per-page kernel."""
    rng = np.random.default_rng(11)
    words = np.array([f"m{i:05d}" + "q" * (i % 7) for i in range(4000)], dtype=object)
    t = pa.table({"s": pa.array(words[rng.integers(0, len(words), 6000)])})
    path = tmp_path / "m.parquet"
    pq.write_table(t, path, compression="snappy", data_page_size=4096)
    first, pages = _emu_run(emu, path, tmp_path)
    assert first.startswith("rows")
    big = [k for k, (_, u, kind) in enumerate(pages) if u >= 200]
    small = [k for k, (_, u, kind) in enumerate(pages) if u < 200]
    if target == "warp" and not small:  # make one: a tiny file of one short page
        t = pa.table({"s": pa.array(["ab", "ab", "abab", "x"] * 3)})
        pq.write_table(t, path, compression="snappy", use_dictionary=False)
        first, pages = _emu_run(emu, path, tmp_path)
        small = [k for k, (_, u, kind) in enumerate(pages) if u < 200]
    k = (big if target == "chain" else small)[0]
    data = np.fromfile(path, dtype=np.uint8)
    i = pages[k][0]
    while data[i] & 0x80:
        i += 1
    data[i + 1] = 0x01
    data[i + 2] = 0x05
    data.tofile(path)
    first, _ = _emu_run(emu, path, tmp_path)
    assert first == f"error 1 {k}", first
