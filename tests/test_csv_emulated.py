"""The device CSV reader's per-record code run on the CPU against the oracle.

The quoting automaton, the field walk and the conversions of
legate-dataframe_b200/csrc/csv.cu are compiled as host C++ with
tests/host_emulation/csv_emu.cpp (a sequential driver that splits records
with the same automaton) under AddressSanitizer, and every case is compared
with the reference's CPU reader, Arrow's CSV reader (CSVRead::cpu_variant,
csv.cpp:58-130), with the options the library's csv_read uses: the same rows,
values (floats bit for bit), nulls, and the same inputs rejected.  The record
split of the GPU path (chunk maps composed by scans) is checked by the GPU
tests in tests/test_csv_gpu.py."""

import io
import math
import shutil
import struct
import subprocess
from pathlib import Path

import numpy as np
import pyarrow as pa
import pyarrow.csv as pacsv
import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "legate-dataframe_b200" / "csrc" / "csv.cu"
EMU = ROOT / "tests" / "host_emulation" / "csv_emu.cpp"

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")

LDF = {pa.bool_(): 1, pa.int8(): 2, pa.int16(): 3, pa.int32(): 4, pa.int64(): 5, pa.uint8(): 6, pa.uint16(): 7,
       pa.uint32(): 8, pa.uint64(): 9, pa.float32(): 10, pa.float64(): 11, pa.string(): 12}
NULLS = list(pacsv.ConvertOptions().null_values)


def _sections() -> str:
    src = SRC.read_text()
    a = src[src.index("constexpr int kCsvMaxCols"):src.index("// ---- 1. records")]
    b = src[src.index("// ---- 3. field conversions"):src.index("// Field count of the first non-empty record")]
    return a + "\n" + b


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    d = tmp_path_factory.mktemp("csv_emu")
    (d / "csv_sections.inc").write_text(_sections())
    subprocess.run(["python", str(ROOT / "legate-dataframe_b200" / "csrc" / "pow5_table.py"), str(d / "pow5_table.inc")],
                   check=True)
    exe = d / "csv_emu"
    cmd = ["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
           f"-I{ROOT / 'include'}", f"-I{d}", str(EMU), "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return exe


def run_emu(exe, text: bytes, cols, header: bool, na: bool, delim=","):
    """cols: [(field index, arrow type)].  Returns ("error", code) or a list of columns of python values."""
    nulls = NULLS if na else []
    head = f"{ord(delim)} {1 if header else 0} {len(cols)} {len(nulls)}\n"
    head += "".join(f"{f} {LDF[t]}\n" for f, t in cols)
    head += "".join(s + "\n" for s in nulls)
    r = subprocess.run([str(exe)], input=head.encode() + text, capture_output=True)
    assert r.returncode == 0, r.stderr.decode()[-3000:]
    lines = r.stdout.decode().splitlines()
    if lines[0].startswith("error"):
        return ("error", int(lines[0].split()[1]))
    rows = int(lines[0].split()[1])
    out, k = [], 1
    for _, t in cols:
        vals = []
        for line in lines[k:k + rows]:
            if line == "N":
                vals.append(None)
            elif line.startswith("S "):
                vals.append(bytes.fromhex(line[2:]).decode("utf-8"))
            elif line.startswith("F "):
                bits = int(line[2:], 16)
                vals.append(struct.unpack("<f" if t == pa.float32() else "<d",
                                          struct.pack("<I" if t == pa.float32() else "<Q", bits))[0])
            elif t == pa.bool_():
                vals.append(bool(int(line[2:])))
            else:
                vals.append(int(line[2:]))
        out.append(vals)
        k += rows
    return out


def header_names(text: bytes, delim: str):
    """Names of the first non-empty line (the tests' headers hold no quotes)."""
    for line in text.replace(b"\r\n", b"\n").replace(b"\r", b"\n").split(b"\n"):
        if line:
            return pacsv.read_csv(io.BytesIO(line + b"\n"), parse_options=pacsv.ParseOptions(delimiter=delim)).schema.names
    return []


def run_arrow(text: bytes, cols, header: bool, na: bool, delim=","):
    if header:
        ropt = pacsv.ReadOptions()
        names = header_names(text, delim)
        include = [names[f] for f, _ in cols]
    else:
        ropt = pacsv.ReadOptions(autogenerate_column_names=True)
        include = [f"f{f}" for f, _ in cols]
    conv = pacsv.ConvertOptions(column_types={n: t for n, (_, t) in zip(include, cols)}, include_columns=include,
                                strings_can_be_null=na, quoted_strings_can_be_null=na)
    if not na:
        conv.null_values = []
    try:
        t = pacsv.read_csv(io.BytesIO(text), read_options=ropt, parse_options=pacsv.ParseOptions(delimiter=delim),
                           convert_options=conv)
    except (pa.ArrowInvalid, pa.ArrowNotImplementedError):
        return ("error", None)
    return [t.column(n).to_pylist() for n in include]


def same(a, b) -> bool:
    if isinstance(a, tuple) or isinstance(b, tuple):
        return isinstance(a, tuple) and isinstance(b, tuple)
    if len(a) != len(b):
        return False
    for x, y in zip(a, b):
        if len(x) != len(y):
            return False
        for u, v in zip(x, y):
            if isinstance(u, float) and isinstance(v, float):
                if math.isnan(u) and math.isnan(v):
                    continue
                if struct.pack("<d", u) != struct.pack("<d", v):
                    return False
            elif u != v:
                return False
    return True


def check(exe, text, cols, header=False, na=True, delim=","):
    got = run_emu(exe, text, cols, header, na, delim)
    exp = run_arrow(text, cols, header, na, delim)
    assert same(got, exp), f"text={text[:300]!r} cols={cols}\n got={str(got)[:600]}\n exp={str(exp)[:600]}"


INT_CASES = ["0", "-0", "1", " 1", "1 ", "\t7\t", "01", "00000000000000000000000000042", "+1", "-", "", "NA",
             "0x10", "0X1f", "0xff", "0x", "0xG", "-0x10", "0x00000000000000001", "0x7fffffffffffffff",
             "0x8000000000000000", "0xffffffffffffffff", "1e3", "1.0", "- 1", "--1", "  ", "127", "128", "-128",
             "-129", "255", "256", "32767", "32768", "-32769", "65535", "65536", "2147483647", "2147483648",
             "-2147483648", "-2147483649", "4294967295", "4294967296", "9223372036854775807", "9223372036854775808",
             "-9223372036854775808", "-9223372036854775809", "18446744073709551615", "18446744073709551616", "null",
             "nan", "x1", "1x", '"12"', '"NA"', '""', '" 5 "']
FLOAT_CASES = ["1.5", ".5", "5.", ".", "1e", "1e5", "1E+5", "1e-5", " 1.5", "2.5\t", "inf", "-inf", "Inf", "INF",
               "infinity", "-Infinity", "InFiNiTy", "infin", "nan", "NaN", "NAN", "-nan", "+1.5", "1,5", "0x1p3",
               "1e400", "1e-400", "-0.0", "0", "-0", '"2.5"', "1.5f", "1_000", "1 .5", "00.5", "1e+05", "1E-0",
               "-.5", "+.5", "1.e5", ".e5", "1.5e", "1.5e+", "123456789012345678901234567890",
               "0.000000000000000000000000000001234567890123456789", "-", "+", "e5", "1e5.5", "1d5", "-inf ",
               "1e-324", "2.4703282292062328e-324", "2.4703282292062329e-324", "4.9406564584124654e-324",
               "2.2250738585072011e-308", "2.2250738585072014e-308", "1.7976931348623157e308",
               "1.7976931348623158e308", "1.7976931348623159e308", "9007199254740993", "9007199254740992.5",
               "0.1", "0.30000000000000004", "3.4028235e38", "3.4028236e38", "1e-46", "1e-45", "1.4e-45",
               "16777217", "16777216.5", "1.00000006", "1.000000059604644775390625", "7.0064923216240854e-46",
               "1e23", "8.988465674311579e307", "1e999999999", "1e-999999999", "000000000000000000000000000001e0"]
BOOL_CASES = ["true", "True", "TRUE", "1", "0", "false", "False", "FALSE", "yes", "t", "tRUE", " true", "true ",
              "", "NA", '"true"', "2"]
STR_CASES = ["", "NA", '""', '"NA"', "x", '"a""b"', '"ab"c', 'a"b', '"a"b"c"', '"a,b"', ' "a"', '"a" ',
             "café", '"été"', "\U0001F642", "null", "N/A", "a b"]


@pytest.mark.parametrize("typ", [pa.int8(), pa.int16(), pa.int32(), pa.int64(), pa.uint8(), pa.uint16(),
                                 pa.uint32(), pa.uint64()])
@pytest.mark.parametrize("na", [True, False])
def test_integer_fields(emu, typ, na):
    for v in INT_CASES:
        check(emu, f"a,b\n{v},1\n".encode(), [(0, typ)], header=True, na=na)


@pytest.mark.parametrize("typ", [pa.float32(), pa.float64()])
@pytest.mark.parametrize("na", [True, False])
def test_float_fields(emu, typ, na):
    for v in FLOAT_CASES:
        check(emu, f"a,b\n{v},1\n".encode(), [(0, typ)], header=True, na=na)


@pytest.mark.parametrize("na", [True, False])
def test_bool_and_string_fields(emu, na):
    for v in BOOL_CASES:
        check(emu, f"a,b\n{v},1\n".encode(), [(0, pa.bool_())], header=True, na=na)
    for v in STR_CASES:
        check(emu, f"a,b\n{v},1\n".encode(), [(0, pa.string())], header=True, na=na)
    check(emu, b"a,b\n\xff,1\n", [(0, pa.string())], header=True, na=na)  # invalid UTF-8
    check(emu, b"a,b\n\xed\xa0\x80,1\n", [(0, pa.string())], header=True, na=na)  # a surrogate


def test_random_floats_bit_exact(emu):
    """Random decimals of 1-25 significant digits and wide exponents, ties
    between neighbouring floats included, against Arrow bit for bit."""
    rng = np.random.default_rng(5)
    vals = []
    for _ in range(3000):
        nd = int(rng.integers(1, 26))
        digits = "".join(str(d) for d in rng.integers(0, 10, nd))
        e = int(rng.integers(-330, 310))
        sign = "-" if rng.random() < 0.3 else ""
        vals.append(f"{sign}{digits[:1]}.{digits[1:]}e{e}" if nd > 1 else f"{sign}{digits}e{e}")
    for _ in range(500):  # exact midpoints of neighbouring doubles and floats
        x = float(rng.standard_normal() * 10.0 ** rng.integers(-300, 300))
        y = np.nextafter(x, np.inf)
        from decimal import Decimal, getcontext
        getcontext().prec = 800
        vals.append(str((Decimal(x) + Decimal(float(y))) / 2))
        f = np.float32(rng.standard_normal() * 10.0 ** rng.integers(-30, 30))
        g = np.nextafter(f, np.float32(np.inf))
        vals.append(str((Decimal(float(f)) + Decimal(float(g))) / 2))
    body = "\n".join(f"{v},{v}" for v in vals)
    text = ("a,b\n" + body + "\n").encode()
    check(emu, text, [(0, pa.float64()), (1, pa.float32())], header=True, na=False)


def test_records_quotes_and_line_ends(emu):
    S = [(0, pa.string()), (1, pa.string())]
    for text in [b"a,b\r\n1,2\r\n\r\n3,4", b"a,b\n1,2\n   \n3,4\n", b"\n\na,b\n1,2\n", b'a,b\n"x\ny",2\n',
                 b"a,b\n1,2\n3,4\r", b"a,b\n1,2\n\r\n", b"a,b\n1,\n", b"a,b\n", b"a,b\n1,2\r3,4\n",
                 b"a,b\r1,2\r\r3,4", b'a,b\na,"x', b"a,b\na,b,c\n", b"a,b\na\n", b'a,b\n"a\r\nb",c\r\n',
                 b'a,b\n"",""\n', b'a,b\n"a""",b\n', b"a,b\n,\n,\n"]:
        check(emu, text, S, header=True, na=True)
        check(emu, text, S, header=True, na=False)
    check(emu, b"1;2\n3;4\n", [(1, pa.int64()), (0, pa.int64())], header=False, na=True, delim=";")
    check(emu, b"x\ty\n1\t2\n", [(1, pa.int32())], header=True, na=True, delim="\t")


def test_random_tables(emu):
    """Tables written by Arrow (every value quoted or not as its writer
    chooses) read back, with nulls, in both null modes."""
    rng = np.random.default_rng(6)
    n = 2000
    words = np.array(["alpha", "be,ta", 'ga"mma', "", "NA", "délta", "e\nps"], dtype=object)
    t = pa.table({
        "i8": pa.array(rng.integers(-128, 128, n), pa.int8()),
        "u32": pa.array(rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)),
        "i64": pa.array(rng.integers(-2**63, 2**63 - 1, n), mask=rng.random(n) < 0.1),
        "f64": pa.array(rng.standard_normal(n) * 10.0 ** rng.integers(-20, 20, n), mask=rng.random(n) < 0.1),
        "f32": pa.array((rng.standard_normal(n) * 1e3).astype(np.float32)),
        "b": pa.array(rng.random(n) < 0.5, mask=rng.random(n) < 0.1),
        "s": pa.array(words[rng.integers(0, len(words), n)], mask=rng.random(n) < 0.1),
    })
    buf = io.BytesIO()
    pacsv.write_csv(t, buf)
    text = buf.getvalue()
    cols = [(j, t.schema.field(j).type) for j in range(t.num_columns)]
    check(emu, text, cols, header=True, na=True)
    check(emu, text, [(1, pa.uint32()), (6, pa.string())], header=True, na=False)
