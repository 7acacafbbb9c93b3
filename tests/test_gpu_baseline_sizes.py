"""Parity at the benchmark's own sizes, through the C ABI, against the oracle
run on the same seeded inputs:

* 3D convection-diffusion 128^3, Pe 20 (n = 2,097,152; the headline
  workload): every I_k bit-exact, M (plain FP64 form) within 1e-10 of the
  reference-order MGS build, iterations within one of the oracle's, and the
  verified relative residual below 1e-8; the headline m_bf16 form converges
  to the same verified tolerance.
* 2D variable-coefficient diffusion 512^2 (n = 262,144; the differentiation
  workload): forward and adjoint solves against the oracle's.
* the first 64 systems of the 512-system batch (8 right-hand sides each):
  every (system, right-hand side) pair against the oracle on that system.
"""
import numpy as np
import pytest

import oracle
from dcu_b200 import native as N
from dcu_b200 import workloads as W

pytestmark = pytest.mark.gpu

RTOL_M = 1e-10


def _d(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def cd3d128():
    A = W.convdiff3d(128, 20.0)
    b, xt = W.rhs_from_solution(A, seed=7)
    return A, b


def test_cd3d128_pattern_bit_exact(ctx, cd3d128):
    A, _ = cd3d128
    cnt_o, iptr_o, il_o = oracle.pattern(A)
    cnt, iptr, il = ctx.pattern_d(A.n, _d(A.ptr), _d(A.idx))
    assert np.array_equal(cnt.cpu().numpy(), cnt_o)
    assert np.array_equal(iptr.cpu().numpy(), iptr_o)
    assert np.array_equal(il.cpu().numpy(), il_o)


def test_cd3d128_plain_fp64_against_oracle(ctx, cd3d128):
    import torch

    A, b = cd3d128
    m_o, res_o, _, sing = oracle.spai(A, "mgs")
    assert sing == 0
    ref = oracle.bicgstab(A, m_o, b, None, tol=1e-8, tol_mode="rel", maxiter=1000)
    ptr, idx, val, bd = _d(A.ptr), _d(A.idx), _d(A.val), _d(b)
    x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    mval = torch.zeros(A.nnz, dtype=torch.float64, device="cuda")
    bi, si = ctx.solve_d(A.n, A.nnz, ptr, idx, val, bd, x, mval_d=mval, precision=N.PREC_FP64)
    m = mval.cpu().numpy()
    assert bi.cols_total == A.n and bi.cols_singular == 0
    assert _rel(m, m_o) < RTOL_M
    assert si.status == N.SOLVE_CONVERGED
    assert abs(si.iters - ref["iters"]) <= 1, (si.iters, ref["iters"])
    xh = x.cpu().numpy()
    relres = np.linalg.norm(b - A.matvec(xh)) / np.linalg.norm(b)
    assert relres < 1e-8
    # the oracle's own solution and ours agree to the tolerance both met
    assert np.linalg.norm(xh - ref["x"]) / np.linalg.norm(ref["x"]) < 1e-6


def test_cd3d128_headline_form_converges(ctx, cd3d128):
    import torch

    A, b = cd3d128
    ptr, idx, val, bd = _d(A.ptr), _d(A.idx), _d(A.val), _d(b)
    x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    bi, si = ctx.solve_d(A.n, A.nnz, ptr, idx, val, bd, x, precision=N.PREC_M_BF16)
    assert si.status == N.SOLVE_CONVERGED
    relres = np.linalg.norm(b - A.matvec(x.cpu().numpy())) / np.linalg.norm(b)
    assert relres < 1e-8


@pytest.fixture(scope="module")
def varcoef512():
    A = W.varcoef2d(512, seed=5)
    rng = np.random.Generator(np.random.PCG64(5))
    b, xt = rng.standard_normal(A.n), rng.standard_normal(A.n)
    m_o, _, _, sing = oracle.spai(A, "mgs")
    assert sing == 0
    return A, b, xt, m_o


def _transpose(A, mval):
    """A^T as CSC (A's CSR arrays) and M^T's values on A^T's pattern."""
    rp, ri, rv = oracle.csc2csr(A.n, A.ptr, A.idx, A.val)
    _, _, mv = oracle.csc2csr(A.n, A.ptr, A.idx, mval)
    return W.CSC(A.n, rp, ri, rv), mv


def test_varcoef512_forward_and_adjoint(ctx, varcoef512):
    """Forward solve A x = b, then the adjoint A^T lam = 2 (x - x_t) with M^T,
    both against the oracle (the adjoint as the oracle's solve of A^T with M^T
    on A^T's pattern).  The iteration counts here run to several hundred, where
    FP64 rounding in a different summation order moves BiCGSTAB's count: the
    band is the spread the oracle itself shows under last-bit perturbations of
    its preconditioner (tests/golden/sensitivity.json)."""
    import json
    import os

    import torch

    A, b, xt, m_o = varcoef512
    band = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "sensitivity.json")))["varcoef512"]
    ptr, idx, val, bd = _d(A.ptr), _d(A.idx), _d(A.val), _d(b)
    x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    mval = torch.zeros(A.nnz, dtype=torch.float64, device="cuda")
    bi, si = ctx.solve_d(A.n, A.nnz, ptr, idx, val, bd, x, mval_d=mval, precision=N.PREC_FP64, maxiter=3000)
    m = mval.cpu().numpy()
    assert _rel(m, m_o) < RTOL_M
    ref = oracle.bicgstab(A, m_o, b, None, tol=1e-8, tol_mode="rel", maxiter=3000)
    assert si.status == N.SOLVE_CONVERGED and ref["status"] == 0
    assert abs(si.iters - ref["iters"]) <= band["forward_iters_band"], (si.iters, ref["iters"])
    xh = x.cpu().numpy()
    assert np.linalg.norm(b - A.matvec(xh)) / np.linalg.norm(b) < 1e-8
    # adjoint
    g = 2.0 * (xh - xt)
    lam = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    ai = ctx.bicgstab_transpose_d(A.n, A.nnz, ptr, idx, val, mval, _d(g), lam, maxiter=3000)
    At, mt = _transpose(A, m_o)
    ref_t = oracle.bicgstab(At, mt, g, None, tol=1e-8, tol_mode="rel", maxiter=3000)
    assert ai.status == N.SOLVE_CONVERGED and ref_t["status"] == 0
    assert abs(ai.iters - ref_t["iters"]) <= band["adjoint_iters_band"], (ai.iters, ref_t["iters"])
    lh = lam.cpu().numpy()
    assert np.linalg.norm(g - At.matvec(lh)) / np.linalg.norm(g) < 1e-8
    assert np.linalg.norm(lh - ref_t["x"]) / np.linalg.norm(ref_t["x"]) < 1e-5


def _block(A, s0, s1):
    sub_ptr = A.ptr[s0:s1 + 1] - A.ptr[s0]
    sub_idx = A.idx[A.ptr[s0]:A.ptr[s1]] - s0
    sub_val = A.val[A.ptr[s0]:A.ptr[s1]]
    return W.CSC(s1 - s0, sub_ptr.astype(np.int32), sub_idx.astype(np.int32), sub_val)


def test_batch512_first_64_systems(ctx):
    """The first 64 systems of the 512-system batch, exactly as generated for
    the benchmark (same seed and size distribution), solved as one batch.
    Every pair's count within the spread the oracle itself shows when M moves
    by one ulp (tests/golden/sensitivity.json: 44 of the 512 pairs move, by
    up to 3 iterations)."""
    import json
    import os

    import torch

    band = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "sensitivity.json")))[
        "batch512_first64"]["iters_band"]
    bt = W.batch_systems()
    ns = 64
    off = bt.offsets[: ns + 1].astype(np.int64)
    A = _block(bt.A, 0, int(off[-1]))
    B = np.ascontiguousarray(bt.B[: off[-1]])
    nrhs = B.shape[1]
    X = torch.zeros((A.n, nrhs), dtype=torch.float64, device="cuda")
    mval = torch.zeros(A.nnz, dtype=torch.float64, device="cuda")
    iters, status, bi, si = ctx.batch_solve_d(_d(off.astype(np.int32)), A.n, A.nnz, _d(A.ptr), _d(A.idx),
                                              _d(A.val), _d(B), X, mval_d=mval)
    assert (status == N.SOLVE_CONVERGED).all(), status
    Xh, m_all = X.cpu().numpy(), mval.cpu().numpy()
    worst = 0
    for s in range(ns):
        s0, s1 = int(off[s]), int(off[s + 1])
        As = _block(A, s0, s1)
        m_s, _, _, _ = oracle.spai(As, "mgs")
        assert _rel(m_all[A.ptr[s0]:A.ptr[s1]], m_s) <= RTOL_M
        for q in range(nrhs):
            b = B[s0:s1, q]
            ref = oracle.bicgstab(As, m_s, b, None, tol=1e-8, tol_mode="rel", maxiter=1000)
            x = Xh[s0:s1, q]
            assert np.linalg.norm(b - As.matvec(x)) / np.linalg.norm(b) < 1e-8
            worst = max(worst, abs(int(iters[s, q]) - ref["iters"]))
    assert worst <= band, (worst, band)
