"""The span that the look-ahead L2 bulk prefetch (cp.async.bulk.prefetch.L2 in
legate-dataframe_b200/csrc/common.cuh) asks for, checked on the CPU: the
helper `prefetch_span` is compiled as host C++ and run on random buffer
addresses and byte ranges.  The span must start on a 16-byte boundary, have a
size that is a multiple of 16, lie inside the requested bytes [lo, hi) of the
buffer (so no prefetch reaches memory outside the array it was issued for),
and miss fewer than 16 bytes at either end."""

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
COMMON = ROOT / "legate-dataframe_b200" / "csrc" / "common.cuh"

DRIVER = r"""
#include <cstdint>
#include <cstdio>
#include <random>
#define __host__
#define __device__
#define __forceinline__ inline
#include "span.inc"

int main()
{
  std::mt19937_64 rng(12345);
  long checked = 0, empty = 0;
  for (int it = 0; it < 400000; ++it) {
    // buffers at any alignment (1, 2, 4, 8 or 16 bytes, or none) and ranges
    // from empty to a few MB, including ranges near 2^32 bytes
    const int align = 1 << (rng() % 5);
    const uint64_t b0 = ((rng() & 0xffffffffffull) + 0x100000000ull) & ~uint64_t(align - 1);
    int64_t lo = static_cast<int64_t>(rng() % (it % 7 == 0 ? (1ull << 33) : 5000000));
    int64_t len = static_cast<int64_t>(rng() % (it % 5 == 0 ? 64 : (it % 11 == 0 ? (1ull << 33) : 3000000)));
    if (it % 13 == 0) len = 0;
    const int64_t hi = lo + len;
    uint64_t a = 0;
    const uint32_t bytes = prefetch_span(b0, lo, hi, &a);
    if (bytes == 0) {
      // nothing asked, or no whole 16-byte block inside, or over the size field
      const uint64_t first = (b0 + lo + 15) & ~15ull, last = (b0 + hi) & ~15ull;
      if (hi > lo && last > first && last - first <= 0xfffffff0ull) {
        std::printf("FAIL empty span for b0=%llx lo=%lld hi=%lld\n", (unsigned long long)b0, (long long)lo,
                    (long long)hi);
        return 1;
      }
      ++empty;
      continue;
    }
    const bool ok = (a % 16 == 0) && (bytes % 16 == 0) && a >= b0 + lo && a + bytes <= b0 + hi &&
                    a - (b0 + lo) < 16 && (b0 + hi) - (a + bytes) < 16;
    if (!ok) {
      std::printf("FAIL b0=%llx lo=%lld hi=%lld a=%llx bytes=%u\n", (unsigned long long)b0, (long long)lo,
                  (long long)hi, (unsigned long long)a, bytes);
      return 1;
    }
    ++checked;
  }
  std::printf("ok %ld spans, %ld empty\n", checked, empty);
  return 0;
}
"""


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


def test_prefetch_span_stays_inside_the_buffer(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    span = _func(COMMON.read_text(), "__host__ __device__ __forceinline__ uint32_t prefetch_span")
    (tmp_path / "span.inc").write_text(span)
    (tmp_path / "driver.cpp").write_text(DRIVER)
    exe = tmp_path / "driver"
    subprocess.run([gxx, "-std=c++17", "-O2", "-fsanitize=address,undefined", f"-I{tmp_path}",
                    str(tmp_path / "driver.cpp"), "-o", str(exe)], check=True, capture_output=True, text=True)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    assert res.stdout.startswith("ok"), res.stdout
