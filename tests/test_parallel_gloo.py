"""Column-sharded SPAI build over 2 and 3 ranks (gloo, CPU): the split
follows the reference's distributeColumns and the all-gather of the ranks'
contiguous slices assembles exactly the single-process M.  The per-rank
column build here is the CPU oracle (there is no GPU in this test); the
library's device builder runs the same sharded_build in
tests/test_gpu_sharded.py."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, schedule, result_path):
    import torch
    import torch.distributed as dist

    import oracle
    from dcu_b200 import parallel
    from dcu_b200 import workloads as W

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        A = W.circuit_like()
        oracle.set_threads(1)

        def build(start, end):
            m, _, _, _ = oracle.spai(A, "mgs", start, end)
            return torch.from_numpy(np.ascontiguousarray(m[A.ptr[start]:A.ptr[end]]))

        m = parallel.sharded_build(build, A.ptr, A.n, rank, world, schedule)
        s, e = parallel.column_range(A.ptr, A.n, rank, world, schedule)
        np.save(f"{result_path}.{rank}.npy", np.concatenate([[s, e], m.numpy()]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,schedule", [(2, 0), (2, 1), (3, 1)])
def test_sharded_build_ranks(tmp_path, world, schedule):
    import torch.multiprocessing as mp

    import oracle
    from dcu_b200 import workloads as W

    port = _free_port()
    path = str(tmp_path / "m")
    mp.start_processes(_worker, args=(world, port, schedule, path), nprocs=world, start_method="spawn", join=True)
    A = W.circuit_like()
    full, _, _, _ = oracle.spai(A, "mgs")
    res = [np.load(f"{path}.{r}.npy") for r in range(world)]
    # the ranks cover [0, n) in order without overlap
    assert res[0][0] == 0 and res[-1][1] == A.n
    assert all(res[r][1] == res[r + 1][0] for r in range(world - 1))
    for r in range(world):
        assert np.array_equal(res[r][2:], full)
