"""Batched systems x right-hand sides (the batching config, small): every
(system, rhs) pair against the oracle run on that system alone."""
import numpy as np
import pytest

import oracle
from dcu_b200 import native as N
from dcu_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _block(A, s0, s1):
    sub_ptr = A.ptr[s0:s1 + 1] - A.ptr[s0]
    sub_idx = A.idx[A.ptr[s0]:A.ptr[s1]] - s0
    sub_val = A.val[A.ptr[s0]:A.ptr[s1]]
    return W.CSC(s1 - s0, sub_ptr.astype(np.int32), sub_idx.astype(np.int32), sub_val)


@pytest.mark.parametrize("nrhs", [8, 1])
def test_batch_matches_single_systems(ctx, nrhs):
    import torch

    bt = W.batch_systems(count=6, nrhs=nrhs, n_lo=200, n_hi=3000, seed=9)
    A = bt.A
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    X = torch.zeros((A.n, nrhs), dtype=torch.float64, device="cuda")
    mval = torch.zeros(A.nnz, dtype=torch.float64, device="cuda")
    iters, status, bi, si = ctx.batch_solve_d(d(bt.offsets.astype(np.int32)), A.n, A.nnz, d(A.ptr), d(A.idx),
                                              d(A.val), d(bt.B), X, mval_d=mval)
    assert (status == N.SOLVE_CONVERGED).all(), status
    Xh = X.cpu().numpy()
    m_all = mval.cpu().numpy()
    for s in range(len(bt.offsets) - 1):
        s0, s1 = int(bt.offsets[s]), int(bt.offsets[s + 1])
        As = _block(A, s0, s1)
        m_s, _, _, _ = oracle.spai(As, "mgs")
        assert np.max(np.abs(m_all[A.ptr[s0]:A.ptr[s1]] - m_s)) <= 1e-10 * np.max(np.abs(m_s))
        for q in range(nrhs):
            b = bt.B[s0:s1, q]
            ref = oracle.bicgstab(As, m_s, b, None, tol=1e-8, tol_mode="rel", maxiter=1000)
            x = Xh[s0:s1, q]
            assert np.linalg.norm(b - As.matvec(x)) / np.linalg.norm(b) < 1e-8
            assert abs(int(iters[s, q]) - ref["iters"]) <= 1, (s, q, iters[s, q], ref["iters"])


def test_batch_rejects_coupled_blocks(ctx):
    import torch

    from dcu_b200.api import DcuError

    A = W.convdiff2d(16, 1.0)  # one coupled matrix, split into two "systems"
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    off = np.array([0, 100, A.n], dtype=np.int32)
    X = torch.zeros((A.n, 2), dtype=torch.float64, device="cuda")
    B = torch.ones((A.n, 2), dtype=torch.float64, device="cuda")
    with pytest.raises(DcuError):
        ctx.batch_solve_d(d(off), A.n, A.nnz, d(A.ptr), d(A.idx), d(A.val), B, X)
