"""The multi-rank exchange on the GPU path: `repartition_by_hash` with the
local hash_partition kernel and NCCL all-to-alls, as a one-rank job on one
GPU (the exchange is then the rank's send to itself).  The
rank must get back every row, in the oracle's bucket order: rows of bucket 0
... of the only rank, input order within each."""

import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

SCRIPT = r'''
import os, sys
sys.path[:0] = [sys.argv[1], sys.argv[1] + "/legate-dataframe_b200"]
from datetime import timedelta
import numpy as np, pyarrow as pa, torch, torch.distributed as dist
from legate_dataframe import LogicalTable
from legate_dataframe.lib.shuffle import repartition_by_hash
from oracle import relational as R
torch.cuda.set_device(0)
dist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=60),
                        device_id=torch.device("cuda", 0))
rng = np.random.default_rng(7)
n = 100_000
t = pa.table({"k": pa.array(rng.integers(0, 1000, n), mask=rng.random(n) < 0.05),
              "s": pa.array([None if m else f"v{x}" * (x % 3) for x, m in zip(rng.integers(0, 90, n), rng.random(n) < 0.1)]),
              "x": rng.normal(size=n)})
got = repartition_by_hash(LogicalTable.from_arrow(t), ["k"]).to_arrow()
exp, _, _ = R.hash_partition(t, ["k"], 1)
dist.destroy_process_group()
assert got.num_rows == n
for c in exp.column_names:
    assert got.column(c).combine_chunks().equals(exp.column(c).combine_chunks()), c
print("exchange ok")
'''


def test_repartition_by_hash_nccl_one_rank():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), NCCL_NVLS_ENABLE="0")
    res = subprocess.run([sys.executable, "-c", SCRIPT, str(ROOT)], capture_output=True, text=True, timeout=300,
                         env=env, cwd=ROOT)
    assert res.returncode == 0 and "exchange ok" in res.stdout, res.stderr[-3000:]
