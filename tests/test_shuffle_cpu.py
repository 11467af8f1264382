"""The multi-rank exchange after the local hash partition
(lib.shuffle.repartition_by_hash, the step of the reference's
task::repartition_by_hash shuffle, cpp/src/core/repartition_by_hash.cu:
146-262) with the gloo backend at world size 2 and 3 on CPU: every rank ends
with exactly the rows of all ranks whose key hashes to its bucket, in
source-rank order and input order inside a bucket, fixed-width, nullable
and string columns alike.  The local partition step is the oracle's here
(the kernel needs a GPU); the exchange plan, sizes and transfers are the
product code."""

import os
import socket
import traceback
from datetime import timedelta

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _local_table(rank: int, n: int):
    import numpy as np
    import pyarrow as pa

    rng = np.random.default_rng(100 + rank)
    k = pa.array(rng.integers(0, 500, n), mask=rng.random(n) < 0.05, type=pa.int64())
    v = pa.array(rng.normal(size=n), mask=rng.random(n) < 0.1, type=pa.float64())
    s = pa.array([None if m else f"r{rank}s{x}" * (x % 4) for x, m in zip(rng.integers(0, 50, n), rng.random(n) < 0.1)],
                 type=pa.string())
    i = rng.integers(-5, 5, n).astype(np.int32)
    return pa.table({"k": k, "v": v, "s": s, "i": i})


def _worker(rank, world, port, sizes, q):
    try:
        import sys
        from pathlib import Path

        root = Path(__file__).resolve().parents[1]
        for p in (str(root), str(root / "legate-dataframe_b200")):
            if p not in sys.path:
                sys.path.insert(0, p)
        import pyarrow as pa
        import torch
        import torch.distributed as dist

        from legate_dataframe import LogicalTable
        from legate_dataframe.lib.shuffle import repartition_by_hash
        from oracle import relational as R

        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
        cpu = torch.device("cpu")

        def oracle_partition(tbl, keys, nparts):
            t, offsets, _ = R.hash_partition(tbl.to_arrow(), keys, nparts)
            return LogicalTable.from_arrow(t, device=cpu), offsets

        local = _local_table(rank, sizes[rank])
        got = repartition_by_hash(LogicalTable.from_arrow(local, device=cpu), ["k"], partition=oracle_partition)
        got = got.to_arrow()
        parts = []
        for src in range(world):
            t, offs, _ = R.hash_partition(_local_table(src, sizes[src]), ["k"], world)
            parts.append(t.slice(offs[rank], offs[rank + 1] - offs[rank]))
        exp = pa.concat_tables(parts)
        ok = got.num_rows == exp.num_rows and all(
            got.column(c).combine_chunks().equals(exp.column(c).combine_chunks().cast(got.schema.field(c).type))
            for c in exp.column_names)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, "ok" if ok else f"mismatch: {got.num_rows} rows, expected {exp.num_rows}"))
    except Exception:  # noqa: BLE001 - reported to the parent
        q.put((rank, traceback.format_exc()))


@pytest.mark.parametrize("world,sizes", [(2, [3000, 1700]), (3, [0, 2500, 900])])
def test_repartition_by_hash_gloo(world, sizes):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, sizes, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == {r: "ok" for r in range(world)}, res
