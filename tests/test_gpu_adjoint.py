"""Differentiation: the adjoint BiCGSTAB with M^T and the sampled outer
product, through the torch.autograd binding over the C ABI, against an FP64
dense-solve reference gradient and central finite differences on 32 seeded
directions (2D variable-coefficient diffusion with upwind advection)."""
import numpy as np
import pytest

from dcu_b200 import native as N
from dcu_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = dict(tol=1e-13, tol_mode=N.TOL_REL, maxiter=2000)


def _setup(m=32, seed=5):
    import torch

    A = W.varcoef2d(m, seed=seed, corr=4.0)
    rng = np.random.Generator(np.random.PCG64(seed))
    b = rng.standard_normal(A.n)
    xt = rng.standard_normal(A.n)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return A, d(A.ptr), d(A.idx), d(A.val), d(b), d(xt)


def _loss(val, b, xt, ptr, idx, ctx):
    from dcu_b200.autograd import spai_solve

    x = spai_solve(val, b, ptr, idx, ctx, **TOL)
    return ((x - xt) ** 2).sum()


def test_transpose_solve(ctx):
    import torch

    A, ptr, idx, val, b, _ = _setup()
    m = torch.zeros_like(val)
    x = torch.zeros_like(b)
    ctx.solve_d(A.n, A.nnz, ptr, idx, val, b, x, mval_d=m, **TOL)
    lam = torch.zeros_like(b)
    info = ctx.bicgstab_transpose_d(A.n, A.nnz, ptr, idx, val, m, b, lam, **TOL)
    assert info.status == N.SOLVE_CONVERGED
    Ad = A.to_scipy().toarray()
    ref = np.linalg.solve(Ad.T, b.cpu().numpy())
    assert np.max(np.abs(lam.cpu().numpy() - ref)) <= 1e-9 * np.max(np.abs(ref))


def test_gradient_vs_dense_reference(ctx):
    A, ptr, idx, val, b, xt = _setup()
    val = val.clone().requires_grad_(True)
    b = b.clone().requires_grad_(True)
    L = _loss(val, b, xt, ptr, idx, ctx)
    L.backward()
    Ad = A.to_scipy().toarray()
    x = np.linalg.solve(Ad, b.detach().cpu().numpy())
    lam = np.linalg.solve(Ad.T, 2.0 * (x - xt.cpu().numpy()))
    cols = np.repeat(np.arange(A.n), np.diff(A.ptr))
    gA = -lam[A.idx] * x[cols]
    assert np.max(np.abs(b.grad.cpu().numpy() - lam)) <= 1e-8 * np.max(np.abs(lam))
    assert np.max(np.abs(val.grad.cpu().numpy() - gA)) <= 1e-8 * np.max(np.abs(gA))


def test_gradient_central_differences_32_directions(ctx):
    import torch

    A, ptr, idx, val, b, xt = _setup()
    v0 = val.clone().requires_grad_(True)
    b0 = b.clone().requires_grad_(True)
    L = _loss(v0, b0, xt, ptr, idx, ctx)
    L.backward()
    gv, gb = v0.grad.detach(), b0.grad.detach()
    rng = np.random.Generator(np.random.PCG64(32))
    for _ in range(32):
        dv = torch.from_numpy(rng.standard_normal(A.nnz)).cuda() * val.abs()   # relative perturbation of A's values
        db = torch.from_numpy(rng.standard_normal(A.n)).cuda()
        h = 1e-6
        with torch.no_grad():
            lp = _loss(val + h * dv, b + h * db, xt, ptr, idx, ctx).item()
            lm = _loss(val - h * dv, b - h * db, xt, ptr, idx, ctx).item()
        fd = (lp - lm) / (2 * h)
        an = (gv * dv).sum().item() + (gb * db).sum().item()
        assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (fd, an)
