"""The column-sharded build with the library's device builder: two gloo
ranks on one GPU (their build kernels are independent of each other; the
all-gather runs on the host), each building its distributeColumns range with
dcu_spai_build_d.  The assembled M must equal one whole build bit for bit:
every column's arithmetic is fixed by its own data."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, schedule, precision, result_path):
    import torch
    import torch.distributed as dist

    from dcu_b200 import parallel
    from dcu_b200 import workloads as W
    from dcu_b200.api import Context

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        A = W.convdiff3d(24, 20.0)
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        with Context(0) as ctx:
            build = parallel.device_slice_builder(ctx, A.n, A.nnz, d(A.ptr), d(A.idx), d(A.val), A.ptr,
                                                  precision=precision)
            m = parallel.sharded_build(build, A.ptr, A.n, rank, world, schedule)
            np.save(f"{result_path}.{rank}.npy", m.cpu().numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("schedule,precision", [(0, 0), (1, 0), (1, 4)])
def test_sharded_device_build_two_ranks(tmp_path, schedule, precision):
    import torch
    import torch.multiprocessing as mp

    from dcu_b200 import workloads as W
    from dcu_b200.api import Context

    port = _free_port()
    path = str(tmp_path / "m")
    mp.start_processes(_worker, args=(2, port, schedule, precision, path), nprocs=2, start_method="spawn",
                       join=True)
    A = W.convdiff3d(24, 20.0)
    with Context(0) as ctx:
        whole, _, _ = ctx.build_h(A, precision=precision)
    for r in range(2):
        assert np.array_equal(np.load(f"{path}.{r}.npy"), whole)
