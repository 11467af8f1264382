"""The task bodies that wire libldf_b200.so into legate-dataframe
(tests/integration/task_bodies.cpp) type-check against include/ldf_b200.h
and against stand-in declarations of the reference's task-side API
(PhysicalTable::release, TaskMemoryResource, argument::get_next_*, legate
stores), and every C++ block of INTEGRATION.md is an excerpt of that file, so
the documented integration cannot drift from either interface unnoticed."""

import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
BODIES = ROOT / "tests" / "integration" / "task_bodies.cpp"
CUDA_INC = Path("/usr/local/cuda/include")

pytestmark = pytest.mark.skipif(shutil.which("g++") is None or not (CUDA_INC / "cuda_runtime_api.h").exists(),
                                reason="needs g++ and the CUDA runtime headers")


def _syntax_check(src: Path) -> subprocess.CompletedProcess:
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Werror", f"-I{ROOT / 'include'}",
           f"-I{ROOT / 'tests' / 'integration'}", f"-I{CUDA_INC}", str(src)]
    return subprocess.run(cmd, capture_output=True, text=True)


def test_task_bodies_type_check():
    r = _syntax_check(BODIES)
    assert r.returncode == 0, r.stderr


def test_type_check_catches_a_changed_signature(tmp_path):
    """The check is not vacuous: a call with one argument missing fails."""
    bad = tmp_path / "bad.cpp"
    text = BODIES.read_text()
    call = "static_cast<int32_t>(keys.size()), nulls_at_end ? 1 : 0, stable ? 1 : 0, limit, res.data(),"
    assert call in text
    bad.write_text(text.replace(call, "static_cast<int32_t>(keys.size()), nulls_at_end ? 1 : 0, limit, res.data(),"))
    r = _syntax_check(bad)
    assert r.returncode != 0 and "ldf_b200_sort" in r.stderr


def _norm(s: str) -> str:
    return re.sub(r"\s+", " ", s).strip()


def test_integration_doc_blocks_are_excerpts():
    doc = (ROOT / "INTEGRATION.md").read_text()
    blocks = re.findall(r"```cpp\n(.*?)```", doc, flags=re.S)
    assert blocks, "INTEGRATION.md has no C++ blocks"
    body = _norm(BODIES.read_text())
    for b in blocks:
        assert _norm(b) in body, f"INTEGRATION.md block not in task_bodies.cpp:\n{b[:200]}"
