"""Column-sharded SPAI build across ranks (one process per GPU).

The reference splits M's columns over DCUs with distributeColumns
(src/spai_multi_dcu.cpp:1356-1449) and gathers the slices on rank 0 with MPI
(aggregateResults, :2021-2165).  Here every rank builds the columns of its
split on its own GPU, and one all-gather assembles M on every rank: the
ranks' column ranges are contiguous and in rank order, so in A's CSC order
each rank's values are one contiguous slice [ptr[start], ptr[end]).  The
slices are padded to the longest one for the collective (NCCL on GPUs; gloo
on the host, where CUDA slices are staged through host memory), so a rank
moves about nnz values in all, against 2 nnz for an all-reduce of
zero-padded full arrays.
"""
from __future__ import annotations

import numpy as np

from . import native as N
from .api import distribute_columns


def column_range(ptr: np.ndarray, n: int, rank: int, world: int, schedule: int = N.SCHED_BALANCED_COLUMNS):
    """[start, end) of this rank: the reference's split of [0, n) over `world` units."""
    s, e = distribute_columns(ptr, 0, n, world, schedule)
    return int(s[rank]), int(e[rank])


def slice_bounds(ptr: np.ndarray, n: int, world: int, schedule: int = N.SCHED_BALANCED_COLUMNS):
    """Per rank, the [lo, hi) positions of its values in A's CSC order."""
    s, e = distribute_columns(ptr, 0, n, world, schedule)
    return [(int(ptr[a]), int(ptr[b])) for a, b in zip(s, e)]


def sharded_build(build_slice, ptr: np.ndarray, n: int, rank: int, world: int,
                  schedule: int = N.SCHED_BALANCED_COLUMNS, group=None):
    """M's nnz values on every rank.  build_slice(start, end) returns this
    rank's values for columns [start, end): a 1-D float64 tensor of length
    ptr[end] - ptr[start] (on its GPU, or on the host)."""
    import torch
    import torch.distributed as dist

    start, end = column_range(ptr, n, rank, world, schedule)
    mine = build_slice(start, end)
    bounds = slice_bounds(ptr, n, world, schedule)
    assert mine.numel() == bounds[rank][1] - bounds[rank][0]
    if world == 1:
        return mine
    longest = max(hi - lo for lo, hi in bounds)
    stage = (dist.get_backend(group) == "gloo" and mine.is_cuda)
    dev = torch.device("cpu") if stage else mine.device
    send = torch.zeros(max(1, longest), dtype=torch.float64, device=dev)
    send[: mine.numel()] = mine.to(dev)
    recv = torch.empty(world * send.numel(), dtype=torch.float64, device=dev)
    dist.all_gather_into_tensor(recv, send, group=group)
    nnz = int(ptr[n])
    m = torch.empty(nnz, dtype=torch.float64, device=dev)
    for r, (lo, hi) in enumerate(bounds):
        m[lo:hi] = recv[r * send.numel(): r * send.numel() + (hi - lo)]
    return m.to(mine.device) if stage else m


def device_slice_builder(ctx, n, nnz, ptr_d, idx_d, val_d, ptr_h: np.ndarray, **opt):
    """build_slice for sharded_build running libdcu_spai on this rank's GPU
    (dcu_spai_build_d over the rank's column range; its values are the slice
    [ptr[start], ptr[end]) of the returned full-length array)."""
    import torch

    full = torch.zeros(nnz, dtype=torch.float64, device=ptr_d.device)

    def build(start, end):
        ctx.build_d(n, nnz, ptr_d, idx_d, val_d, full, col_start=start, col_end=end, **opt)
        return full[int(ptr_h[start]):int(ptr_h[end])]

    return build
