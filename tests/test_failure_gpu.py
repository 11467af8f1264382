"""Failure handling on the GPU without a fault: a bounded device-side wait is
made to run out (a look-back whose predecessor status word nothing writes),
the call returns LDF_ERR_TIMEOUT, Python raises RuntimeError as the
reference's task bodies raise std::runtime_error, and the next ops on the
same GPU still run and match the oracle."""

import ctypes

import numpy as np
import pyarrow as pa
import pytest

from ldf_testing import assert_tables_equal
from oracle import relational as R

pytestmark = pytest.mark.gpu


def test_expired_wait_reports_timeout_and_the_gpu_stays_usable():
    import torch

    from legate_dataframe import LogicalTable
    from legate_dataframe import _native as N
    from legate_dataframe.lib.groupby_aggregation import groupby_aggregation

    L = N.lib()
    alloc = N.TorchAllocator(N.require_cuda())
    stream = ctypes.c_void_p(N.current_stream_handle())
    for limit in (1, 1000):
        status = L.ldf_b200_test_stalled_lookback(limit, ctypes.byref(alloc.struct), stream)
        assert status == N.LDF_ERR_TIMEOUT
        with pytest.raises(RuntimeError, match="bounded device-side wait expired"):
            N.check(status)
    with pytest.raises(ValueError):
        N.check(L.ldf_b200_test_stalled_lookback(0, ctypes.byref(alloc.struct), stream))
    torch.cuda.synchronize()
    # the context is intact: a groupby that uses the same scan still matches
    rng = np.random.default_rng(3)
    n = 300_000
    t = pa.table({"k": rng.integers(0, 5000, n), "v": pa.array(rng.normal(size=n), mask=rng.random(n) < 0.1)})
    aggs = [("v", "sum", "s"), (None, "count_all", "c"), ("v", "count_distinct", "nd")]
    res = groupby_aggregation(LogicalTable.from_arrow(t), ["k"], aggs).to_arrow()
    assert_tables_equal(res, R.groupby(t, ["k"], aggs), sort_by=["k"], rtol=1e-12)
