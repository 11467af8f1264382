"""The hash partition entry point that allocates no device memory.

It exists for callers that may not allocate device memory themselves (a task
body sharing the GPU with concurrent tasks, where cudaMalloc synchronizes the
device, or a host whose device memory all belongs to its own pool): the
caller hands over the output buffers and the library uses one fixed scratch
array in its device image.  This test calls it through the C ABI, twice in a
row, and checks each result against the allocating ldf_b200_hash_partition,
and that the device's free memory (cudaMemGetInfo) is the same before and
after a call once the first call has loaded the kernels; it also checks that
an oversized input is rejected.  The file is named to run last, so a failure
here comes after every other test has run.
"""

import ctypes

import numpy as np
import pyarrow as pa
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_partition(tbl, keys, nparts):
    import torch

    from legate_dataframe import LogicalColumn, LogicalTable
    from legate_dataframe import _native as N

    n = tbl.num_rows()
    cols = (N.ldf_column * tbl.num_columns())(*[c.to_c() for c in tbl.get_columns()])
    out = (N.ldf_column * tbl.num_columns())()
    keep = []  # the caller owns every output buffer
    for j, c in enumerate(tbl.get_columns()):
        data = torch.empty(max(n * N.TYPE_WIDTH[c.ldf_type], 16), dtype=torch.uint8, device="cuda")
        valid = torch.empty(max(n, 16), dtype=torch.uint8, device="cuda") if c.nullable() else None
        keep.append((data, valid))
        out[j].data = data.data_ptr()
        out[j].valid = valid.data_ptr() if valid is not None else None
    offsets = (ctypes.c_int64 * (nparts + 1))()
    names = tbl.get_column_name_to_index()
    key_idx = N.int32_array([names[k] for k in keys])
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    status = N.lib().ldf_b200_hash_partition_noalloc(
        cols, tbl.num_columns(), key_idx, len(keys), nparts, out, offsets,
        ctypes.c_void_p(N.current_stream_handle()))
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    N.check(status)
    res = [LogicalColumn(c.arrow_type, out[j].type, out[j].size, keep[j][0], keep[j][1])
           for j, c in enumerate(tbl.get_columns())]
    return LogicalTable(res, tbl.get_column_names()).to_arrow(), list(offsets), free_before - free_after


def _table(seed, n):
    rng = np.random.default_rng(seed)
    return pa.table({
        "k": pa.array(rng.integers(0, 10_000, n), mask=rng.random(n) < 0.03),
        "f": pa.array(rng.normal(size=n), mask=rng.random(n) < 0.1),
        "i": rng.integers(-(2**31), 2**31 - 1, n).astype(np.int32),
        "b": pa.array(rng.random(n) < 0.5),
    })


def test_noalloc_matches_allocating_partition_twice():
    from legate_dataframe import LogicalTable
    from legate_dataframe.lib.hash_partition import hash_partition

    for call, (seed, n, keys, nparts) in enumerate(((1, 300_000, ["k"], 64), (2, 1_000_000, ["k", "i"], 256),
                                                     (3, 1 << 20, ["i"], 200))):
        tbl = LogicalTable.from_arrow(_table(seed, n))
        exp, exp_offs = hash_partition(tbl, keys, nparts)
        got, got_offs, used = _noalloc_partition(tbl, keys, nparts)
        assert got_offs == exp_offs
        assert got.equals(exp.to_arrow())
        if call > 0:  # the first call on the device may load the library's kernels
            assert used == 0, f"device free memory dropped by {used} bytes during the call"


def test_noalloc_rejects_oversized_input():
    import torch

    from legate_dataframe import LogicalColumn, LogicalTable
    from legate_dataframe import _native as N

    n = N.NOALLOC_MAX_ROWS + 1
    col = LogicalColumn.from_torch(torch.zeros(n, dtype=torch.int64, device="cuda"), pa.int64())
    with pytest.raises(ValueError, match="at most"):
        _noalloc_partition(LogicalTable([col], ["k"]), ["k"], 8)
