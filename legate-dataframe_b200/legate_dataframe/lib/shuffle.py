"""repartition_by_hash(): the multi-rank exchange that follows the local
hash_partition, mirroring legate-dataframe's ``task::repartition_by_hash``
(cpp/src/core/repartition_by_hash.cu:264-316) and its ``shuffle``
(:146-262).  Every rank splits its rows into ``world`` buckets with the local
``hash_partition`` (bucket ``b`` of a rank goes to rank ``b``), the bucket
sizes are exchanged, then each column's bytes travel in one all-to-all over
``torch.distributed`` (NCCL on GPUs: grouped send/recv over NVLink; gloo on
CPU).  The result on rank ``r`` is every row, from every rank, whose key
hashes to bucket ``r``: rank 0's rows first, then rank 1's, ..., each in the
order the local partition left them (input order inside a bucket), as the
reference concatenates its chunks in peer order.

The exchange moves whole columns, not packed tables: fixed-width values,
the one-byte null masks and, for strings, per-row lengths plus the
characters in row order (ranges are rebuilt on the receiving side).  No
kernel here reads another GPU's memory; the transfers are NCCL's.
"""

from __future__ import annotations

from typing import Callable, Iterable, Optional

import torch

from legate_dataframe import _native as N
from legate_dataframe.lib.core.column import LogicalColumn
from legate_dataframe.lib.core.table import LogicalTable


def _ranges(col: LogicalColumn) -> torch.Tensor:
    """[n, 2] inclusive char ranges of a string column."""
    n = col.size
    if n == 0:
        return torch.empty((0, 2), dtype=torch.int64, device=col.data.device)
    return col.data[: 16 * n].view(torch.int64).view(n, 2)


def _flat_chars(col: LogicalColumn, lens: torch.Tensor) -> torch.Tensor:
    """The column's characters in row order, `lens[i]` bytes for row i."""
    n = col.size
    total = int(lens.sum()) if n else 0
    if total == 0:
        return torch.empty(0, dtype=torch.uint8, device=col.data.device)
    lo = _ranges(col)[:, 0] - col.chars_base
    start = torch.cumsum(lens, 0) - lens
    row = torch.repeat_interleave(torch.arange(n, device=lens.device), lens)
    pos = torch.arange(total, device=lens.device) - start[row]
    return col.chars[lo[row] + pos]


def _exchange(t: torch.Tensor, send_counts, recv_counts, group) -> torch.Tensor:
    """all-to-all of a 1-D tensor split by element counts."""
    import torch.distributed as dist

    out = torch.empty(int(sum(recv_counts)), dtype=t.dtype, device=t.device)
    dist.all_to_all_single(out, t.contiguous(), [int(x) for x in recv_counts], [int(x) for x in send_counts],
                           group=group)
    return out


def repartition_by_hash(tbl: LogicalTable, keys: Iterable[str], group=None,
                        partition: Optional[Callable] = None) -> LogicalTable:
    """This rank's hash partition of the distributed table whose local part
    is `tbl`.  Every rank of `group` must call it with tables of the same
    columns; `partition(tbl, keys, nparts) -> (table, offsets)` defaults to
    the local ``hash_partition`` kernel."""
    import torch.distributed as dist

    from legate_dataframe.lib.hash_partition import hash_partition

    keys = list(keys)
    world = dist.get_world_size(group)
    part = partition or hash_partition
    ptab, offsets = part(tbl, keys, world)
    cols = ptab.get_columns()
    dev = cols[0].data.device if cols else torch.device("cpu")
    send_rows = torch.tensor([offsets[b + 1] - offsets[b] for b in range(world)], dtype=torch.int64, device=dev)
    recv_rows = torch.empty_like(send_rows)
    dist.all_to_all_single(recv_rows, send_rows, group=group)
    # nullability of each column on any rank (a rank without nulls sends ones)
    nullable = torch.tensor([1 if c.valid is not None else 0 for c in cols], dtype=torch.int32, device=dev)
    if len(cols):
        dist.all_reduce(nullable, op=dist.ReduceOp.MAX, group=group)
    sr, rr = send_rows.tolist(), recv_rows.tolist()
    n_out = int(sum(rr))
    out = []
    for j, c in enumerate(cols):
        n = c.size
        valid = None
        if int(nullable[j]):
            v = c.valid[:n] if c.valid is not None else torch.ones(n, dtype=torch.uint8, device=dev)
            valid = _exchange(v, sr, rr, group)
        if c.ldf_type == N.LDF_STRING:
            rng = _ranges(c)
            lens = (rng[:, 1] - rng[:, 0] + 1).clamp(min=0)
            if c.valid is not None:
                lens = torch.where(c.valid[:n] != 0, lens, torch.zeros_like(lens))
            chars = _flat_chars(c, lens)
            bounds = [0] + torch.cumsum(send_rows, 0).tolist()
            csum = torch.cumsum(lens, 0)
            send_chars = [int(csum[bounds[b + 1] - 1] - (csum[bounds[b] - 1] if bounds[b] > 0 else 0))
                          if bounds[b + 1] > bounds[b] else 0 for b in range(world)]
            recv_chars = torch.empty(world, dtype=torch.int64, device=dev)
            dist.all_to_all_single(recv_chars, torch.tensor(send_chars, dtype=torch.int64, device=dev), group=group)
            rlens = _exchange(lens, sr, rr, group)
            rchars = _exchange(chars, send_chars, recv_chars.tolist(), group)
            start = torch.cumsum(rlens, 0) - rlens
            ranges = torch.stack([start, start + rlens - 1], 1).contiguous()
            out.append(LogicalColumn(c.arrow_type, c.ldf_type, n_out, ranges.view(torch.uint8).reshape(-1), valid,
                                     rchars, 0, rchars.numel()))
        else:
            w = N.TYPE_WIDTH[c.ldf_type]
            data = _exchange(c.data[: n * w], [x * w for x in sr], [x * w for x in rr], group)
            out.append(LogicalColumn(c.arrow_type, c.ldf_type, n_out, data, valid))
    return LogicalTable(out, ptab.get_column_names())
