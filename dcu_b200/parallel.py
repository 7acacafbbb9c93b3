"""Column-sharded SPAI build across ranks (one process per GPU).

The reference splits M's columns over DCUs with distributeColumns
(src/spai_multi_dcu.cpp:1356-1449) and gathers the slices on rank 0 with MPI
(:2172-2328).  Here every rank builds the columns of its split on its own GPU
(dcu_spai_build_d with a column range writes zeros elsewhere), and one
all-reduce (sum) of the nnz-long value array over NCCL assembles M on every
rank: the slices are disjoint, so the sum is exact.
"""
from __future__ import annotations

import numpy as np

from . import native as N
from .api import distribute_columns


def column_range(ptr: np.ndarray, n: int, rank: int, world: int, schedule: int = N.SCHED_BALANCED_COLUMNS):
    """[start, end) of this rank: the reference's split of [0, n) over `world` units."""
    s, e = distribute_columns(ptr, 0, n, world, schedule)
    return int(s[rank]), int(e[rank])


def sharded_build(build_slice, ptr: np.ndarray, n: int, rank: int, world: int,
                  schedule: int = N.SCHED_BALANCED_COLUMNS, group=None):
    """M on every rank.  build_slice(start, end) returns this rank's value
    array (a torch tensor of length nnz, zero outside its columns)."""
    import torch.distributed as dist

    start, end = column_range(ptr, n, rank, world, schedule)
    m = build_slice(start, end)
    if world > 1:
        dist.all_reduce(m, op=dist.ReduceOp.SUM, group=group)
    return m


def device_slice_builder(ctx, n, nnz, ptr_d, idx_d, val_d, **opt):
    """build_slice for sharded_build running libdcu_spai on this rank's GPU."""
    import torch

    def build(start, end):
        m = torch.zeros(nnz, dtype=torch.float64, device=ptr_d.device)
        ctx.build_d(n, nnz, ptr_d, idx_d, val_d, m, col_start=start, col_end=end, **opt)
        return m

    return build
