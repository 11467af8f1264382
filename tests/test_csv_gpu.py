"""The device CSV reader (ldf_b200_csv_read through lib.csv.csv_read) against
the reference's CPU reader, Arrow's CSV reader with the same options
(CSVRead::cpu_variant, csv.cpp:58-130): tables written by Arrow with every
supported type and nulls, both null modes, selection by header name and by
field index, other delimiters, several files, quoted fields that run across
the record split's chunks and scan blocks, a 200 MB file, and the inputs it
must reject."""

import io

import numpy as np
import pyarrow as pa
import pyarrow.csv as pacsv
import pytest

from ldf_testing import assert_tables_equal

pytestmark = pytest.mark.gpu


def arrow_read(paths, names, dtypes, na_filter=True, delimiter=",", usecols=None):
    if usecols is None:
        ropt, include, rename = pacsv.ReadOptions(), names, None
    else:
        ropt, include, rename = pacsv.ReadOptions(autogenerate_column_names=True), [f"f{i}" for i in usecols], names
    conv = pacsv.ConvertOptions(column_types=dict(zip(include, dtypes)), include_columns=include,
                                strings_can_be_null=na_filter, quoted_strings_can_be_null=na_filter)
    if not na_filter:
        conv.null_values = []
    # quoted line ends belong to their field, as in the device reader (and
    # cudf's, which the reference's GPU variant calls); Arrow needs to be told
    # so to keep its parallel block split from cutting such fields
    popt = pacsv.ParseOptions(delimiter=delimiter, newlines_in_values=True)
    tabs = [pacsv.read_csv(p, read_options=ropt, parse_options=popt, convert_options=conv) for p in paths]
    t = pa.concat_tables(tabs) if len(tabs) > 1 else tabs[0]
    return t.rename_columns(rename) if rename else t


def device_read(paths, names, dtypes, **kw):
    from legate_dataframe.lib.csv import csv_read

    return csv_read([str(p) for p in paths], dtypes=dtypes, names=names, **kw).to_arrow()


def random_table(n, seed):
    rng = np.random.default_rng(seed)
    words = np.array(["alpha", "be,ta", 'ga"mma', "", "NA", "délta", "e\nps", "x" * 300, "null"], dtype=object)
    return pa.table({
        "b": pa.array(rng.random(n) < 0.5, mask=rng.random(n) < 0.1),
        "i8": pa.array(rng.integers(-128, 128, n), pa.int8()),
        "i16": pa.array(rng.integers(-2**15, 2**15, n), pa.int16(), mask=rng.random(n) < 0.05),
        "i32": pa.array(rng.integers(-2**31, 2**31, n), pa.int32()),
        "i64": pa.array(rng.integers(-2**63, 2**63 - 1, n), mask=rng.random(n) < 0.1),
        "u8": pa.array(rng.integers(0, 256, n), pa.uint8()),
        "u16": pa.array(rng.integers(0, 2**16, n), pa.uint16()),
        "u32": pa.array(rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)),
        "u64": pa.array(rng.integers(0, 2**63, n, dtype=np.uint64) * 2 + 1),
        "f32": pa.array((rng.standard_normal(n) * 10.0 ** rng.integers(-30, 30, n)).astype(np.float32)),
        "f64": pa.array(rng.standard_normal(n) * 10.0 ** rng.integers(-300, 300, n), mask=rng.random(n) < 0.1),
        "s": pa.array(words[rng.integers(0, len(words), n)], mask=rng.random(n) < 0.1),
    })


@pytest.mark.parametrize("na_filter", [True, False])
def test_csv_types_and_nulls(tmp_path, na_filter):
    t = random_table(20_000, 1)
    p = tmp_path / "t.csv"
    pacsv.write_csv(t, p)
    names, dtypes = t.column_names, [f.type for f in t.schema]
    if not na_filter:  # without null spellings, only the columns Arrow can read back without nulls
        keep = [j for j, c in enumerate(t.columns) if c.null_count == 0 or pa.types.is_string(c.type)]
        names, dtypes = [names[j] for j in keep], [dtypes[j] for j in keep]
    exp = arrow_read([p], names, dtypes, na_filter=na_filter)
    got = device_read([p], names, dtypes, na_filter=na_filter)
    assert_tables_equal(got, exp, sort_by=None)


def test_csv_selection_delimiters_and_files(tmp_path):
    t = random_table(5_000, 2)
    paths = []
    for k in range(3):
        p = tmp_path / f"p{k}.csv"
        pacsv.write_csv(t.slice(k * 1000, 1700), p, write_options=pacsv.WriteOptions(delimiter="|"))
        paths.append(p)
    names, dtypes = ["s", "f64", "i8"], [pa.string(), pa.float64(), pa.int8()]
    got = device_read(paths, names, dtypes, delimiter="|")
    assert_tables_equal(got, arrow_read(paths, names, dtypes, delimiter="|"), sort_by=None)
    # no header: fields by index, named by the caller
    nh = tmp_path / "nh.csv"
    pacsv.write_csv(t.slice(0, 3000), nh, write_options=pacsv.WriteOptions(include_header=False, delimiter="\t"))
    got = device_read([nh], ["x", "y"], [pa.int64(), pa.string()], usecols=[4, 11], delimiter="\t")
    exp = arrow_read([nh], ["x", "y"], [pa.int64(), pa.string()], usecols=[4, 11], delimiter="\t")
    assert_tables_equal(got, exp, sort_by=None)


def test_csv_quoted_fields_across_chunks_and_blocks(tmp_path):
    """Quoted fields of up to 400 KB with newlines, carriage returns and
    doubled quotes: they span many 256-byte chunks and several 256 KB scan
    blocks of the record split, so each chunk's start state comes from the
    composition of the maps before it."""
    rng = np.random.default_rng(3)
    rows = []
    for i in range(300):
        ln = int(rng.choice([1, 10, 300, 5_000, 400_000], p=[0.3, 0.3, 0.2, 0.15, 0.05]))
        body = "".join(rng.choice(list('ab\n\r,"'), size=ln))
        rows.append((i, body))
    text = "k,v\r\n" + "".join(f'{i},"{b.replace(chr(34), chr(34) * 2)}"\r\n' for i, b in rows)
    p = tmp_path / "q.csv"
    p.write_bytes(text.encode())
    got = device_read([p], ["k", "v"], [pa.int32(), pa.string()])
    exp = arrow_read([p], ["k", "v"], [pa.int32(), pa.string()])
    assert got.num_rows == 300
    assert_tables_equal(got, exp, sort_by=None)


def test_csv_200mb_file(tmp_path):
    """About 200 MB of CSV: thousands of scan blocks."""
    rng = np.random.default_rng(4)
    n = 3_000_000
    t = pa.table({"k": rng.integers(0, 10**12, n), "x": rng.standard_normal(n),
                  "s": pa.array(np.char.mod("w%07d", rng.integers(0, 10**7, n)).astype(object)),
                  "i": pa.array(rng.integers(-1000, 1000, n), pa.int32(), mask=rng.random(n) < 0.02)})
    p = tmp_path / "big.csv"
    pacsv.write_csv(t, p)
    assert p.stat().st_size > 100e6
    dtypes = [pa.int64(), pa.float64(), pa.string(), pa.int32()]
    got = device_read([p], t.column_names, dtypes)
    assert_tables_equal(got, arrow_read([p], t.column_names, dtypes), sort_by=None)


@pytest.mark.parametrize("text,dtypes", [
    (b"a,b\n1,2\n3\n", [pa.int64(), pa.int64()]),          # a record with too few fields
    (b"a,b\n1,2\n3,4,5\n", [pa.int64(), pa.int64()]),      # too many
    (b"a,b\n1,x\n", [pa.int64(), pa.int64()]),              # not an integer
    (b"a,b\n1,300\n", [pa.int64(), pa.int8()]),             # out of range
    (b"a,b\n1,1.5.5\n", [pa.int64(), pa.float64()]),        # not a float
    (b"a,b\n1,maybe\n", [pa.int64(), pa.bool_()]),          # not a Boolean
    (b"a,b\n1,\xff\n", [pa.int64(), pa.string()]),          # not UTF-8
])
def test_csv_rejects_what_arrow_rejects(tmp_path, text, dtypes):
    p = tmp_path / "bad.csv"
    p.write_bytes(text)
    with pytest.raises(pa.ArrowInvalid):
        arrow_read([p], ["a", "b"], dtypes)
    with pytest.raises(ValueError):
        device_read([p], ["a", "b"], dtypes)


def test_csv_empty_and_header_only(tmp_path):
    e = tmp_path / "e.csv"
    e.write_bytes(b"")
    h = tmp_path / "h.csv"
    h.write_bytes(b"a,b\n")
    got = device_read([e, h], ["a", "b"], [pa.int64(), pa.string()])
    assert got.num_rows == 0
    r = tmp_path / "r.csv"
    r.write_bytes(b"a,b\n5,x")  # no final line end
    got = device_read([h, r], ["b", "a"], [pa.string(), pa.int64()])
    assert got.to_pydict() == {"b": ["x"], "a": [5]}
