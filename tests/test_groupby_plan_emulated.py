"""The partitioned groupby plan's device code (one fixed-width key; hot keys
in shared memory, cold rows routed to hash buckets) run on the CPU: the
plan's section of legate-dataframe_b200/csrc/groupby.cu is compiled as host
C++ with tests/host_emulation/groupby_plan_emu.cpp (CUDA built-ins as host
functions, one thread per block) under AddressSanitizer, then run on skewed
and uniform keys with null keys and nullable values, with the bucket pass at
its real shared-memory capacity and at a reduced one that sends buckets to
the deferred and large (global work memory) paths.  Every group's COUNT(*),
COUNT, SUM, MEAN, MIN, MAX and NUNIQUE (both modes) is compared with a direct
per-key computation.  This checks index arithmetic and plan logic without a
GPU; thread races are outside its reach (the GPU parity tests cover them)."""

import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "legate-dataframe_b200" / "csrc" / "groupby.cu"
EMU = ROOT / "tests" / "host_emulation" / "groupby_plan_emu.cpp"


def _func(src: str, sig: str) -> str:
    i = src.index(sig)
    k = src.index("{", i)
    depth = 0
    while True:
        if src[k] == "{":
            depth += 1
        elif src[k] == "}":
            depth -= 1
            if depth == 0:
                return src[i:k + 1] + "\n"
        k += 1


def _section(small: bool) -> str:
    src = SRC.read_text()
    helpers = src[src.index("struct AggOut {"):src.index("};", src.index("struct AggOut {")) + 2] + "\n"
    for sig in ("__device__ __forceinline__ bool fixed_parts", "__device__ __forceinline__ double chunks_to_double",
                "__device__ __forceinline__ void sh_add_chunk", "__device__ __forceinline__ void sh_add_magnitude",
                "__device__ __forceinline__ void store_double", "__device__ __forceinline__ void store_int",
                "__device__ __forceinline__ uint64_t unordered_bits"):
        helpers += _func(src, sig)
    start = src.rfind("// ====", 0, src.index("// Partitioned plan: one fixed-width key"))
    end = src.index("bool try_partitioned(")
    end += len(_func(src, "bool try_partitioned("))
    sec = src[start:end]
    sec = sec.replace("extern __shared__ __align__(16) unsigned char smem[];", "unsigned char* smem = emu_smem;")
    sec = re.sub(r"__shared__ ", "static ", sec)
    if small:  # a bucket pass that holds 64 groups / ~1,000 rows in shared memory
        for old, new in (("kBucketRecBytes = 96 * 1024;", "kBucketRecBytes = 8 * 1024;"),
                         ("kBucketKeySlots = 1024;", "kBucketKeySlots = 128;"),
                         ("kBucketGroupsMax = 768;", "kBucketGroupsMax = 64;")):
            assert old in sec, old
            sec = sec.replace(old, new)
    return helpers + sec


@pytest.fixture(scope="module")
def emulators(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    out = {}
    d = tmp_path_factory.mktemp("gb_emu")
    for small in (False, True):
        (d / "section.inc").write_text(_section(small))
        exe = d / ("emu_small" if small else "emu")
        cmd = [gxx, "-std=c++17", "-O1", "-g", "-fsanitize=address", "-fno-omit-frame-pointer", "-w",
               f"-I{d}", f"-I{ROOT / 'include'}", str(EMU), "-o", str(exe)]
        subprocess.run(cmd, check=True, capture_output=True, text=True)
        out[small] = exe
    return out


@pytest.mark.parametrize("small", [False, True])
@pytest.mark.parametrize("n,groups", [(600_000, 50_000), (2_000_000, 2_000), (300_000, 200), (500_000, 300_000),
                                      (100_000, 5), (2_500_000, 100_000)])
def test_partitioned_plan_on_host(emulators, small, n, groups):
    res = subprocess.run([str(emulators[small]), str(n), str(groups)], capture_output=True, text=True, timeout=300,
                         env={"ASAN_OPTIONS": "detect_leaks=0"})
    assert res.returncode == 0, res.stderr[-3000:]
    assert "partitioned=1" in res.stdout, res.stdout
    m = re.search(r"aggregate mismatches (\d+) of (\d+) groups", res.stdout)
    assert m and m.group(1) == "0" and int(m.group(2)) > 0, res.stdout
