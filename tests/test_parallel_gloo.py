"""Column-sharded SPAI build over 2 ranks (gloo, CPU): the split follows the
reference's distributeColumns and the all-reduce assembles exactly the
single-process M.  The per-rank column build here is the CPU oracle (there is
no GPU in this test); on GPUs dcu_b200.parallel.device_slice_builder plugs in
the library."""
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
            full = np.zeros(A.nnz)
            full[A.ptr[start]:A.ptr[end]] = m[A.ptr[start]:A.ptr[end]]
            return torch.from_numpy(full)

        m = parallel.sharded_build(build, A.ptr, A.n, rank, world, schedule)
        s, e = parallel.column_range(A.ptr, A.n, rank, world, schedule)
        np.save(f"{result_path}.{rank}.npy", np.concatenate([[s, e], m.numpy()]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("schedule", [0, 1])
def test_sharded_build_two_ranks(tmp_path, schedule):
    import torch.multiprocessing as mp

    import oracle
    from dcu_b200 import workloads as W

    port = _free_port()
    path = str(tmp_path / "m")
    mp.start_processes(_worker, args=(2, port, schedule, path), nprocs=2, start_method="spawn", join=True)
    A = W.circuit_like()
    full, _, _, _ = oracle.spai(A, "mgs")
    r0 = np.load(path + ".0.npy")
    r1 = np.load(path + ".1.npy")
    # the two ranks cover [0, n) without overlap
    assert r0[0] == 0 and r0[1] == r1[0] and r1[1] == A.n
    assert np.array_equal(r0[2:], r1[2:])
    assert np.array_equal(r0[2:], full)
