"""Edge cases through the C ABI: malformed CSC input is refused before any
kernel follows its indices, sizes beyond the limits are refused, and
degenerate systems end with a status (never a hang)."""
import ctypes as C

import numpy as np
import pytest

from dcu_b200 import native as N
from dcu_b200 import workloads as W
from dcu_b200.api import _p

pytestmark = pytest.mark.gpu


def _build_raw(ctx, n, nnz, ptr, idx, val):
    """dcu_spai_build_h with explicit sizes (the arrays hold exactly nnz entries)."""
    o = N.default_options()
    mval = np.zeros(max(1, nnz), dtype=np.float64)
    info = N.BuildInfo()
    return ctx._L.dcu_spai_build_h(ctx.h, n, nnz, _p(ptr), _p(idx), _p(val), C.byref(o), _p(mval), None,
                                   C.byref(info))


def _malformed():
    A = W.convdiff2d(8, 1.0)
    n, nnz = A.n, A.nnz
    out = {}
    p = A.ptr.copy()
    p[5], p[6] = p[6], p[5]                     # ptr decreases
    out["ptr_decreasing"] = (p, A.idx.copy())
    p = A.ptr.copy()
    p[-1] = nnz - 1                             # ptr[n] != nnz
    out["ptr_end"] = (p, A.idx.copy())
    p = A.ptr.copy()
    p[0] = 1                                    # ptr[0] != 0
    out["ptr_start"] = (p, A.idx.copy())
    i = A.idx.copy()
    i[7] = n                                    # row index past the last row
    out["row_too_large"] = (A.ptr.copy(), i)
    i = A.idx.copy()
    i[3] = -1                                   # negative row index
    out["row_negative"] = (A.ptr.copy(), i)
    return n, nnz, A.val.copy(), out


@pytest.mark.parametrize("case", ["ptr_decreasing", "ptr_end", "ptr_start", "row_too_large", "row_negative"])
def test_malformed_csc_is_refused(ctx, case):
    n, nnz, val, cases = _malformed()
    ptr, idx = cases[case]
    rc = _build_raw(ctx, n, nnz, ptr.astype(np.int32), idx.astype(np.int32), val)
    assert rc == N.ERR_ARG, rc
    assert b"malformed" in ctx._L.dcu_spai_last_error(ctx.h)
    # the context stays usable
    A = W.convdiff2d(8, 1.0)
    m, _, info = ctx.build_h(A)
    assert info.cols_total == A.n and np.isfinite(m).all()


def test_sizes_beyond_the_limits_are_refused(ctx):
    tiny = np.zeros(2, dtype=np.int32)
    assert _build_raw(ctx, (1 << 26) - 1, 0, tiny, tiny, np.zeros(1)) == N.ERR_LIMIT
    assert _build_raw(ctx, 0, 0, tiny, tiny, np.zeros(1)) == N.ERR_ARG
    assert _build_raw(ctx, 4, -1, tiny, tiny, np.zeros(1)) == N.ERR_ARG


def test_one_by_one_and_zero_rhs(ctx):
    A = W.CSC(1, np.array([0, 1], np.int32), np.array([0], np.int32), np.array([2.0]))
    x, m, _, si = ctx.solve_h(A, np.array([4.0]), want_m=True)
    assert si.status == N.SOLVE_CONVERGED and x[0] == pytest.approx(2.0) and m[0] == pytest.approx(0.5)
    B = W.convdiff2d(16, 1.0)
    x, _, _, si = ctx.solve_h(B, np.zeros(B.n))       # x0 = 0 already solves b = 0
    assert si.status == N.SOLVE_CONVERGED and si.iters == 1 and not x.any()


def test_empty_matrix_ends_in_breakdown(ctx):
    # every column empty: M = 0, A y = 0, so (r*, A y) = 0 in the first step
    n = 64
    A = W.CSC(n, np.zeros(n + 1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    x, _, bi, si = ctx.solve_h(A, np.ones(n))
    assert si.status == N.SOLVE_BREAKDOWN and bi.cols_total == n


def test_non_finite_values_end_in_breakdown(ctx):
    A = W.convdiff2d(16, 1.0)
    val = A.val.copy()
    val[10] = np.nan
    An = W.CSC(A.n, A.ptr, A.idx, val)
    x, _, _, si = ctx.solve_h(An, np.ones(A.n))
    assert si.status == N.SOLVE_BREAKDOWN
    # and the next, finite solve on the same context is unaffected
    b, _ = W.rhs_from_solution(A, seed=1)
    x, _, _, si = ctx.solve_h(A, b)
    assert si.status == N.SOLVE_CONVERGED and np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b) < 1e-8


def _duplicated():
    """Matrices whose column holds one row index twice: adjacent in a sorted
    column, apart in an unsorted one, and 40 places apart in a long unsorted
    column (past one warp's 32 entries)."""
    from tests.test_gpu_pattern import random_csc

    out = {}
    A = W.convdiff2d(8, 1.0)
    p = int(A.ptr[10])
    i = A.idx.copy()
    i[p + 1] = i[p]
    out["sorted_adjacent"] = (A, i)
    i = A.idx.copy()
    r0, r1, r2 = (int(v) for v in A.idx[p:p + 3])
    i[p:p + 3] = [r1, r2, r1]
    out["unsorted_apart"] = (A, i)
    B = random_csc(300, 0.3, 5)                 # ~90 entries per column, shuffled
    c = int(np.argmax(np.diff(B.ptr)))
    q = int(B.ptr[c])
    i = B.idx.copy()
    i[q + 45] = i[q + 5]
    out["long_unsorted"] = (B, i)
    return out


@pytest.mark.parametrize("case", ["sorted_adjacent", "unsorted_apart", "long_unsorted"])
def test_duplicate_rows_are_refused(ctx, case):
    import torch

    A, idx = _duplicated()[case]
    rc = _build_raw(ctx, A.n, A.nnz, A.ptr.astype(np.int32), idx.astype(np.int32), A.val.copy())
    assert rc == N.ERR_ARG, rc
    assert b"same row index twice" in ctx._L.dcu_spai_last_error(ctx.h)
    # the format conversion accepts the pair, as the reference's does
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    rp = torch.zeros(A.n + 1, dtype=torch.int32, device="cuda")
    ri = torch.zeros(A.nnz, dtype=torch.int32, device="cuda")
    rv = torch.zeros(A.nnz, dtype=torch.float64, device="cuda")
    ctx.csc_to_csr_d(A.n, A.nnz, d(A.ptr), d(idx.astype(np.int32)), d(A.val), rp, ri, rv)
    assert int(rp[-1].item()) == A.nnz
    # and the same matrix without the repeat, in shuffled order, builds
    m, _, info = ctx.build_h(A)
    assert info.cols_total == A.n and np.isfinite(m).all()
