"""Build recipe of libldf_b200.so: every CUDA source compiled by nvcc for
sm_100a and linked into one C-ABI shared library inside the package
(``legate_dataframe/libldf_b200.so``), so it travels with the source tree.

Usage: ``python legate-dataframe_b200/build.py [--force] [--verbose]``.
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG_ROOT = Path(__file__).resolve().parent
REPO_ROOT = PKG_ROOT.parent
CSRC = PKG_ROOT / "csrc"
INCLUDE = REPO_ROOT / "include"
BUILD_DIR = REPO_ROOT / "_build" / "csrc"
LIB = PKG_ROOT / "legate_dataframe" / "libldf_b200.so"

SOURCES = [
    "runtime.cu",
    "table_ops.cu",
    "join.cu",
    "groupby.cu",
    "radix.cu",
    "sort.cu",
    "abi.cu",
    "noalloc.cu",
    "batch.cu",
    "distinct.cu",
    "ingest.cu",
    "csv.cu",
    "parquet.cu",
]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC,-O3",
    f"-I{INCLUDE}",
    f"-I{BUILD_DIR}",  # generated tables (pow5_table.inc)
]


def _newest_input_mtime() -> float:
    files = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.py")) + list(INCLUDE.glob("*.h"))
    files.append(Path(__file__))
    return max(f.stat().st_mtime for f in files)


def _compile(src: str, verbose: bool) -> Path:
    obj = BUILD_DIR / (src + ".o")
    cmd = [NVCC, *ARCH, *CFLAGS, "-c", str(CSRC / src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    if verbose:
        sys.stderr.write(res.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile (if stale) and return the path of libldf_b200.so."""
    if LIB.exists() and not force and LIB.stat().st_mtime >= _newest_input_mtime():
        sys.stderr.write(f"[ldf_b200 build] {LIB.name} is newer than every source: not recompiled\n")
        return LIB
    BUILD_DIR.mkdir(parents=True, exist_ok=True)
    subprocess.run([sys.executable, str(CSRC / "pow5_table.py"), str(BUILD_DIR / "pow5_table.inc")], check=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC, *ARCH, "-shared", "-o", str(tmp), *map(str, objs)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB)
    sys.stderr.write(f"[ldf_b200 build] compiled {len(objs)} CUDA sources for sm_100a into {LIB.name}\n")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
