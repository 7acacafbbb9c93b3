"""SPAI build (gather + Householder QR + solve + scatter) against the oracle."""
import numpy as np
import pytest

import oracle
from dcu_b200 import native as N
from dcu_b200 import workloads as W
from tests.test_gpu_pattern import random_csc

pytestmark = pytest.mark.gpu

RTOL_FP64 = 1e-10   # M values, FP64 form, relative to max |M| of the column set
RTOL_FP32 = 2e-4    # FP32 least squares


def rel_err(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("name,A", [
    ("cd2d_64", W.convdiff2d(64, 10.0)),
    ("cd3d_16", W.convdiff3d(16, 20.0)),
    ("circuit", W.circuit_like()),
    ("varcoef_32", W.varcoef2d(32, seed=3)),
])
def test_spai_fp64_matches_oracle(ctx, name, A):
    m_o, res_o, E_o, sing_o = oracle.spai(A, "mgs")
    m_h, _, _, _ = oracle.spai(A, "householder")
    m, res, info = ctx.build_h(A)
    assert info.cols_total == A.n
    assert info.cols_small + info.cols_large == A.n
    assert info.cols_singular == sing_o == 0
    assert rel_err(m, m_h) < RTOL_FP64
    assert rel_err(m, m_o) < RTOL_FP64
    assert np.max(np.abs(res - res_o)) < 1e-10


def test_schedules_identical(ctx):
    A = W.circuit_like()
    m0, r0, _ = ctx.build_h(A, schedule=N.SCHED_BALANCED_COLUMNS)
    m1, r1, _ = ctx.build_h(A, schedule=N.SCHED_BALANCED_NNZ)
    assert np.array_equal(m0, m1)
    assert np.array_equal(r0, r1)


def test_column_range_zero_outside(ctx):
    A = W.convdiff2d(32, 10.0)
    s, e = 100, 777
    m, res, info = ctx.build_h(A, col_start=s, col_end=e)
    m_o, res_o, _, _ = oracle.spai(A, "mgs", s, e)
    assert info.cols_total == e - s
    assert rel_err(m, m_o) < RTOL_FP64
    assert np.all(m[: A.ptr[s]] == 0) and np.all(m[A.ptr[e]:] == 0)


def test_spai_fp32(ctx):
    A = W.convdiff3d(16, 20.0)
    m_o, _, _, _ = oracle.spai(A, "householder")
    m, _, info = ctx.build_h(A, precision=N.PREC_MIXED_FP32)
    assert rel_err(m, m_o) < RTOL_FP32


def test_spai_random_unsorted_and_empty(ctx):
    A = random_csc(300, 0.02, 5, empty_cols=4)
    m_h, res_h, _, sing = oracle.spai(A, "householder")
    m, res, info = ctx.build_h(A)
    ok = np.isfinite(m_h)
    # columns whose least-squares problem is rank deficient give inf/nan on both sides
    assert info.cols_singular == sing
    good_cols = [k for k in range(A.n) if np.all(np.isfinite(m_h[A.ptr[k]:A.ptr[k + 1]]))]
    for k in good_cols:
        a, b = m[A.ptr[k]:A.ptr[k + 1]], m_h[A.ptr[k]:A.ptr[k + 1]]
        if len(b):
            assert np.max(np.abs(a - b)) <= 1e-8 * max(1.0, np.max(np.abs(b))), k
    assert ok.sum() > 0


@pytest.mark.parametrize("units", [1, 3, 1000])
def test_static_units_identical(units):
    from dcu_b200.api import Context

    A = W.convdiff3d(12, 20.0)
    with Context(0) as c0, Context(0, units=units) as c1:
        m0, r0, _ = c0.build_h(A)
        m1, r1, _ = c1.build_h(A)
        assert c1.units == units
    assert np.array_equal(m0, m1) and np.array_equal(r0, r1)


@pytest.mark.parametrize("ls", [N.LS_AUTO, N.LS_HOUSEHOLDER])
@pytest.mark.parametrize("name,A", [("cd3d_16", W.convdiff3d(16, 20.0)), ("circuit", W.circuit_like()),
                                    ("cd2d_64", W.convdiff2d(64, 10.0))])
def test_spai_fp32_methods(ctx, ls, name, A):
    """FP32 least squares: thread-per-column normal equations (with hand-off
    to Householder) and Householder alone both match the FP64 oracle."""
    m_h, res_h, _, _ = oracle.spai(A, "householder")
    m, res, info = ctx.build_h(A, precision=N.PREC_MIXED_BF16, ls_method=ls)
    assert info.cols_small + info.cols_large == A.n
    assert info.cols_singular == 0
    for k in range(A.n):   # per column, relative to the column's own scale
        a, b = m[A.ptr[k]:A.ptr[k + 1]], m_h[A.ptr[k]:A.ptr[k + 1]]
        if len(b):
            assert np.max(np.abs(a - b)) <= RTOL_FP32 * 10 * np.max(np.abs(b)), (k, a, b)
    assert np.max(np.abs(res - res_h)) < 1e-3


@pytest.mark.parametrize("name,A", [("cd3d_16", W.convdiff3d(16, 20.0)), ("circuit", W.circuit_like()),
                                    ("cd2d_64", W.convdiff2d(64, 10.0))])
def test_spai_fp64_normal_equations(ctx, name, A):
    """FP64 normal equations (hand-off below pivot ratio 1e-8) against the FP64 oracle."""
    m_h, res_h, _, _ = oracle.spai(A, "householder")
    m, res, info = ctx.build_h(A, precision=N.PREC_FP64, ls_method=N.LS_NORMAL_EQ)
    assert info.cols_small + info.cols_large == A.n
    assert rel_err(m, m_h) < 1e-9


def test_bulk_copy_staging_matches_plain_loads(ctx):
    """The CTA kernel stages its J columns in shared memory with bulk (TMA)
    copies when A's arrays are 16-byte aligned, and reads them from global
    memory otherwise; both give the same M, bit for bit, equal to the oracle's
    within 1e-10.  The pattern kernel (no value array) stages indices only."""
    import torch

    A = W.circuit_like()
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    ptr = d(A.ptr)
    idx, val = d(A.idx), d(A.val)
    # the same arrays 4 / 8 bytes past a 16-byte boundary: no bulk copies
    idx_u = torch.empty(A.nnz + 1, dtype=torch.int32, device="cuda")[1:]
    val_u = torch.empty(A.nnz + 1, dtype=torch.float64, device="cuda")[1:]
    idx_u.copy_(idx)
    val_u.copy_(val)
    assert idx_u.data_ptr() % 16 != 0 and val_u.data_ptr() % 16 != 0
    m1 = torch.zeros(A.nnz, dtype=torch.float64, device="cuda")
    m2 = torch.zeros_like(m1)
    i1 = ctx.build_d(A.n, A.nnz, ptr, idx, val, m1)
    i2 = ctx.build_d(A.n, A.nnz, ptr, idx_u, val_u, m2)
    assert i1.cols_large > 0 and i1.cols_staged > 0 and i2.cols_staged == 0
    assert torch.equal(m1, m2)
    m_o, _, _, _ = oracle.spai(A, "mgs")
    mh = m1.cpu().numpy()
    assert np.max(np.abs(mh - m_o)) <= 1e-10 * np.max(np.abs(m_o))
    c1, p1, l1 = ctx.pattern_d(A.n, ptr, idx)
    c2, p2, l2 = ctx.pattern_d(A.n, ptr, idx_u)
    assert torch.equal(c1, c2) and torch.equal(l1, l2)


@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_MIXED_BF16])
def test_hub_kernels_match_one_cta_per_column(prec):
    """Dense blocks larger than a CTA's shared memory (the circuit-like
    matrix's hub columns) are factored by the all-SM hub kernels, one launch
    per Householder step; with cta_max_area = -1 one CTA factors each from a
    global slab, and with a limit in between both paths share the columns.
    All agree with the oracle's Householder to the form's rounding, and the
    hub path is deterministic."""
    from dcu_b200.api import Context

    A = W.circuit_like()
    m_h, res_h, _, _ = oracle.spai(A, "householder")
    with Context(0) as c:
        m0, r0, i0 = c.build_h(A, precision=prec)
        m0b, _, _ = c.build_h(A, precision=prec)
        c.set_tuning(prec, cta_max_area=-1)
        m1, r1, i1 = c.build_h(A, precision=prec)
        c.set_tuning(prec, cta_max_area=200000)
        m2, r2, i2 = c.build_h(A, precision=prec)
    assert i0.cols_hub > 0 and i1.cols_hub == 0 and i2.cols_hub <= i0.cols_hub
    assert i0.cols_large == i1.cols_large == i2.cols_large
    assert np.array_equal(m0, m0b)
    tol = RTOL_FP64 if prec == N.PREC_FP64 else RTOL_FP32 * 10
    for m, r in ((m0, r0), (m1, r1), (m2, r2)):
        for k in range(A.n):
            a, b = m[A.ptr[k]:A.ptr[k + 1]], m_h[A.ptr[k]:A.ptr[k + 1]]
            if len(b):
                assert np.max(np.abs(a - b)) <= tol * np.max(np.abs(b)), (k, prec)
        assert np.max(np.abs(r - res_h)) < (1e-10 if prec == N.PREC_FP64 else 1e-3)


def rank_deficient_hub(n=400, seed=5):
    """Column 0 has rows 1..300 (|J| = 300), and each of those columns has
    three rows among 0..49, so |I_0| <= 50 < |J_0|: a rank-deficient least-
    squares problem whose block (<= 50 x 301) exceeds shared memory."""
    rng = np.random.default_rng(seed)
    cols = [(np.arange(1, 301), rng.standard_normal(300))]
    for _ in range(1, 301):
        cols.append((np.sort(rng.choice(50, 3, replace=False)), rng.standard_normal(3)))
    for j in range(301, n):
        cols.append((np.array([j]), np.array([2.0])))
    ptr = np.zeros(n + 1, np.int32)
    for j, (r, _) in enumerate(cols):
        ptr[j + 1] = ptr[j] + len(r)
    idx = np.concatenate([c[0] for c in cols]).astype(np.int32)
    val = np.concatenate([c[1] for c in cols])
    return W.CSC(n, ptr, idx, val)


def test_hub_column_with_fewer_rows_than_columns(ctx):
    """The hub path on |I| < |J|: the column is reported singular (as by the
    oracle's Householder), R's missing rows are never read, and every other
    column matches the oracle."""
    A = rank_deficient_hub()
    m_h, res_h, _, sing = oracle.spai(A, "householder")
    m, res, info = ctx.build_h(A)
    assert info.cols_hub >= 1 and sing == 1 and info.cols_singular == sing
    assert not np.all(np.isfinite(m[A.ptr[0]:A.ptr[1]]))
    for k in range(1, A.n):
        a, b = m[A.ptr[k]:A.ptr[k + 1]], m_h[A.ptr[k]:A.ptr[k + 1]]
        assert np.max(np.abs(a - b)) <= RTOL_FP64 * max(1.0, np.max(np.abs(b))), k


def test_static_schedule_speed_does_not_depend_on_units():
    """balanced_columns with one unit (one "DCU") must not serialise the build:
    the resident workers sweep the units' ranges together.  (Giving each
    worker its own unit once left all but one worker idle: ~3400x slower at
    128^3 with one unit.)  The bound is loose; the columns are identical."""
    import torch

    from dcu_b200.api import Context

    A = W.convdiff3d(48, 20.0)
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    p, i, v = d(A.ptr), d(A.idx), d(A.val)
    out = {}
    for units in (0, 1, 3):
        with Context(0, units=units) as c:
            for prec in (N.PREC_FP64, N.PREC_M_BF16):
                m = torch.zeros(A.nnz, dtype=torch.float64, device="cuda")
                ms = min(c.build_d(A.n, A.nnz, p, i, v, m, precision=prec).ms for _ in range(3))
                out[(units, prec)] = (ms, m.cpu().numpy())
    for prec in (N.PREC_FP64, N.PREC_M_BF16):
        base_ms, base_m = out[(0, prec)]
        for units in (1, 3):
            ms, m = out[(units, prec)]
            assert np.array_equal(m, base_m)
            assert ms < 5.0 * base_ms + 0.2, (units, prec, ms, base_ms)
