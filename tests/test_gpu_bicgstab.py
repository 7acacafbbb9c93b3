"""BiCGSTAB: iteration count within +-1 of the oracle, residual below tol."""
import numpy as np
import pytest

import oracle
from dcu_b200 import native as N
from dcu_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_config1_reference_settings(ctx):
    # b = 1, x0 = 1, ||r|| < 1e-7 absolute (runBiCGSTABOnRank0)
    A = W.convdiff2d(64, 10.0)
    m_o, _, _, _ = oracle.spai(A, "mgs")
    ref = oracle.bicgstab(A, m_o, np.ones(A.n), np.ones(A.n), tol=1e-7, tol_mode="abs", maxiter=10000)
    m, _, _ = ctx.build_h(A)
    x, info = ctx.bicgstab_h(A, m, np.ones(A.n), np.ones(A.n), tol=1e-7, tol_mode=N.TOL_ABS, maxiter=10000, verify=0)
    assert info.status == N.SOLVE_CONVERGED
    assert abs(info.iters - ref["iters"]) <= 1
    assert ref["iters"] == 43
    assert info.res < 1e-7


@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_MIXED_FP32, N.PREC_MIXED_BF16, N.PREC_M_FP32, N.PREC_M_BF16])
def test_config1_solve(ctx, prec):
    A = W.convdiff2d(64, 10.0)
    b = W.rhs_ones_product(A)
    m_o, _, _, _ = oracle.spai(A, "mgs")
    ref = oracle.bicgstab(A, m_o, b, None, tol=1e-8, tol_mode="rel", maxiter=1000)
    x, _, bi, si = ctx.solve_h(A, b, precision=prec)
    assert si.status == N.SOLVE_CONVERGED
    relres = np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b)
    assert relres < 1e-8
    assert si.true_res / si.bnorm < 1e-8
    if prec == N.PREC_FP64:
        assert abs(si.iters - ref["iters"]) <= 1
    else:
        # a different (rounded) preconditioner / FP32 Krylov vectors: the
        # count may move, the verified residual may not
        assert si.iters <= 1.25 * ref["iters"] + 3
    assert np.max(np.abs(x - 1.0)) < 1e-5


def test_circuit_like(ctx):
    A = W.circuit_like()
    rng = np.random.Generator(np.random.PCG64(11))
    b = rng.uniform(-1, 1, A.n)
    m_o, _, _, _ = oracle.spai(A, "mgs")
    ref = oracle.bicgstab(A, m_o, b, None, tol=1e-8, tol_mode="rel", maxiter=1000)
    x, _, bi, si = ctx.solve_h(A, b)
    assert si.status == N.SOLVE_CONVERGED
    assert abs(si.iters - ref["iters"]) <= 1
    assert np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b) < 1e-8


def test_3d_small(ctx):
    A = W.convdiff3d(24, 20.0)
    b, xt = W.rhs_from_solution(A)
    m_o, _, _, _ = oracle.spai(A, "mgs")
    ref = oracle.bicgstab(A, m_o, b, None, tol=1e-8, tol_mode="rel", maxiter=1000)
    for prec in (N.PREC_FP64, N.PREC_MIXED_BF16):
        x, _, bi, si = ctx.solve_h(A, b, precision=prec)
        assert si.status == N.SOLVE_CONVERGED
        assert np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b) < 1e-8
        if prec == N.PREC_FP64:
            assert abs(si.iters - ref["iters"]) <= 1


def test_maxiter_counter(ctx):
    A = W.convdiff2d(64, 10.0)
    b = W.rhs_ones_product(A)
    m, _, _ = ctx.build_h(A)
    x, info = ctx.bicgstab_h(A, m, b, maxiter=5, tol=1e-30, verify=0)
    assert info.status == N.SOLVE_MAXITER
    assert info.iters == 5   # the reference's counter runs 1..MAX_ITER


def _shuffled_columns(A, seed):
    """Same matrix with each column's entries in a seeded random order."""
    rng = np.random.default_rng(seed)
    idx, val = A.idx.copy(), A.val.copy()
    for c in range(A.n):
        s, e = A.ptr[c], A.ptr[c + 1]
        o = rng.permutation(e - s)
        idx[s:e], val[s:e] = idx[s:e][o], val[s:e][o]
    return W.CSC(A.n, A.ptr, idx, val)


def _one_sided(A):
    """A's pattern with one off-diagonal entry removed: no longer symmetric."""
    c = A.n // 2
    s, e = A.ptr[c], A.ptr[c + 1]
    drop = next(k for k in range(s, e) if A.idx[k] != c)
    keep = np.ones(A.nnz, bool)
    keep[drop] = False
    ptr = A.ptr.copy()
    ptr[c + 1:] -= 1
    return W.CSC(A.n, ptr, A.idx[keep], A.val[keep])


def _empty_columns(A):
    """Symmetric pattern with a whole row/column pair (index 5) emptied."""
    keep = np.ones(A.nnz, bool)
    cols = np.repeat(np.arange(A.n), np.diff(A.ptr))
    keep[(A.idx == 5) | (cols == 5)] = False
    ptr = np.zeros(A.n + 1, np.int32)
    ptr[1:] = np.cumsum(np.bincount(cols[keep], minlength=A.n))
    return W.CSC(A.n, ptr, A.idx[keep], A.val[keep])


CSR_CASES = {
    "circuit": lambda: W.circuit_like(),                              # general path
    "cd2d_64": lambda: W.convdiff2d(64, 10.0),                        # symmetric pattern
    "cd3d_16": lambda: W.convdiff3d(16, 20.0),                        # symmetric pattern
    "cd2d_shuffled": lambda: _shuffled_columns(W.convdiff2d(32, 10.0), 3),  # symmetric, unsorted
    "cd2d_one_sided": lambda: _one_sided(W.convdiff2d(32, 10.0)),     # almost symmetric
    "cd2d_empty": lambda: _empty_columns(W.convdiff2d(32, 10.0)),     # symmetric, empty column
}


@pytest.mark.parametrize("case", list(CSR_CASES))
def test_csr_matches_oracle(ctx, case):
    import torch

    A = CSR_CASES[case]()
    rp_o, ri_o, rv_o = oracle.csc2csr(A.n, A.ptr, A.idx, A.val)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    rp = torch.zeros(A.n + 1, dtype=torch.int32, device="cuda")
    ri = torch.zeros(A.nnz, dtype=torch.int32, device="cuda")
    rv = torch.zeros(A.nnz, dtype=torch.float64, device="cuda")
    ctx.csc_to_csr_d(A.n, A.nnz, d(A.ptr), d(A.idx), d(A.val), rp, ri, rv)
    assert np.array_equal(rp.cpu().numpy(), rp_o)
    assert np.array_equal(ri.cpu().numpy(), ri_o)
    assert np.array_equal(rv.cpu().numpy(), rv_o)


def test_host_path_matches_device_path(ctx):
    """dcu_spai_solve_h (uploads overlapped with the analysis and the build)
    returns exactly what dcu_spai_solve_d returns, from pageable and from
    pinned host buffers, with a nonzero x0."""
    import torch

    A = W.convdiff3d(24, 20.0)
    b, _ = W.rhs_from_solution(A, seed=4)
    x0 = np.random.default_rng(9).standard_normal(A.n) * 1e-3
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    xd = d(x0)
    md = torch.zeros(A.nnz, dtype=torch.float64, device="cuda")
    ctx.solve_d(A.n, A.nnz, d(A.ptr), d(A.idx), d(A.val), d(b), xd, mval_d=md, precision=N.PREC_M_BF16)
    x_dev, m_dev = xd.cpu().numpy(), md.cpu().numpy()

    x_h, m_h, _, si = ctx.solve_h(A, b, x0=x0, want_m=True, precision=N.PREC_M_BF16)
    assert si.status == N.SOLVE_CONVERGED
    assert np.array_equal(x_h, x_dev) and np.array_equal(m_h, m_dev)

    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    hx, hm = pin(x0), pin(np.zeros(A.nnz))
    ctx.solve_h_into(A.n, A.nnz, pin(A.ptr), pin(A.idx), pin(A.val), pin(b), hx, mval=hm, precision=N.PREC_M_BF16)
    assert np.array_equal(hx, x_dev) and np.array_equal(hm, m_dev)


def test_sell_plan_stats_and_offset_aligned_slices(ctx):
    """A 3D stencil lays out in offset-uniform slices (no index reads) except
    where row + offset leaves the matrix; an irregular matrix mostly does not.
    Both solve to the same iterations as the oracle (the layout only moves
    zeros around)."""
    for A, lo, hi, wide in ((W.convdiff3d(16, 20.0), 0.95, 1.0, False), (W.circuit_like(), 0.0, 0.9, True)):
        b, _ = W.rhs_from_solution(A, seed=2)
        x, _, _, si = ctx.solve_h(A, b, precision=N.PREC_FP64)
        slots, uni, nwide = ctx.sell_plan_stats(wide=True)
        assert slots >= A.nnz and 0 <= uni <= slots
        assert lo <= uni / slots <= hi, (uni, slots)
        # the long rows of the circuit-like matrix (hubs of 200-400 entries,
        # power-law degrees) make their slices wide: summed by the
        # warp-cooperative pre-pass
        assert (nwide > 0) == wide, nwide
        m_o, _, _, _ = oracle.spai(A, "mgs")
        ref = oracle.bicgstab(A, m_o, b, None, tol=1e-8, tol_mode="rel", maxiter=1000)
        assert si.status == N.SOLVE_CONVERGED and abs(si.iters - ref["iters"]) <= 1
        assert np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b) < 1e-8


@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_M_BF16])
def test_wide_prepass_keeps_iterates_bit_identical(ctx, prec):
    """The circuit-like matrix's hub rows make wide SELL slices, summed by the
    warp-cooperative pre-pass (each row in its own order, long rows by one
    chain in k order).  With the pre-pass off the SpMV kernels' per-lane loop
    sums the same rows: the iterates and the count must not change by a bit."""
    import torch

    A = W.circuit_like()
    rng = np.random.Generator(np.random.PCG64(11))
    b = rng.uniform(-1, 1, A.n)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    ptr, idx, val, bd = d(A.ptr), d(A.idx), d(A.val), d(b)
    out = []
    try:
        for on in (True, False):
            ctx.set_wide_prepass(on)
            x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
            bi, si = ctx.solve_d(A.n, A.nnz, ptr, idx, val, bd, x, precision=prec)
            _, _, nwide = ctx.sell_plan_stats(wide=True)
            assert (nwide > 0) == on
            assert si.status == N.SOLVE_CONVERGED
            out.append((x.cpu().numpy(), si.iters, si.res))
    finally:
        ctx.set_wide_prepass(True)
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][2] == out[1][2]


def _dyadic_circuit():
    """circuit_like with every value rounded up in magnitude to a multiple of
    1/8: exact in FP32, and its hub rows still make wide slices."""
    A = W.circuit_like()
    v = np.sign(A.val) * np.ceil(np.abs(A.val) * 8.0) / 8.0
    return W.CSC(A.n, A.ptr, A.idx, v)


def _one_value_off():
    """An integer stencil with one value moved by 2^-30: FP32 rounds that one
    value, so the whole matrix must keep the FP64 reads."""
    A = W.convdiff3d(24, 20.0)
    v = A.val.copy()
    v[len(v) // 2] += 2.0 ** -30
    return W.CSC(A.n, A.ptr, A.idx, v)


EXACT_A32_CASES = {
    "stencil3d_integer": (lambda: W.convdiff3d(24, 20.0), 1),
    "circuit_dyadic_wide": (_dyadic_circuit, 1),
    "stencil3d_one_value_off": (_one_value_off, 0),
    "varcoef_inexact": (lambda: W.varcoef2d(64, seed=3), 0),
}


@pytest.mark.parametrize("case", list(EXACT_A32_CASES))
@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_M_BF16])
def test_exact_fp32_a_keeps_iterates_bit_identical(ctx, case, prec):
    """A's FP32 copy is read only when every value of A is exact in FP32, and
    then it holds the same numbers: the iterates, the count and the residuals
    equal those of the FP64 reads bit for bit.  A single value that FP32
    rounds keeps the whole solve on the FP64 reads (a_fp32 = 0); if it did
    not, that value would change and the bits with it.  The plain FP64 form
    never reads the copy."""
    import torch

    make, expect = EXACT_A32_CASES[case]
    if prec == N.PREC_FP64:
        expect = 0
    A = make()
    rng = np.random.Generator(np.random.PCG64(17))
    b = rng.uniform(-1, 1, A.n)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    ptr, idx, val, bd = d(A.ptr), d(A.idx), d(A.val), d(b)
    out = []
    try:
        for on in (True, False):
            ctx.set_exact_a32(on)
            x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
            _, si = ctx.solve_d(A.n, A.nnz, ptr, idx, val, bd, x, precision=prec, maxiter=2000)
            assert si.a_fp32 == (expect if on else 0)
            out.append((x.cpu().numpy(), si.iters, si.status, si.res, si.true_res))
    finally:
        ctx.set_exact_a32(True)
    assert out[0][1:] == out[1][1:]
    assert np.array_equal(out[0][0], out[1][0])
