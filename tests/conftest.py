import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "legate-dataframe_b200"
for p in (str(ROOT), str(PKG), str(Path(__file__).resolve().parent)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests of the sm_100a kernels")


def pytest_collection_modifyitems(config, items):
    import torch

    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this container")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def _built_library():
    """Build libldf_b200.so in-tree when it is missing or stale (nvcc
    cross-compiles here; on a GPU box the prebuilt library travels along)."""
    sys.path.insert(0, str(PKG))
    import build as ldf_build  # legate-dataframe_b200/build.py

    if os.environ.get("LDF_SKIP_BUILD") != "1" or not ldf_build.LIB.exists():
        try:
            ldf_build.build()
        except (RuntimeError, FileNotFoundError):
            if not ldf_build.LIB.exists():
                raise
    from oracle import native as oracle_native

    oracle_native.build()
    yield
