"""The autotuner (dcu_autotune_d) and pinned launch configurations
(dcu_set_tuning): the tuner reports what it timed and keeps its choice; every
iteration setting leaves the solution bit-identical; the warp-group |I| limit
moves columns to the CTA kernel and changes M by rounding only."""
import numpy as np
import pytest

from dcu_b200 import native as N
from dcu_b200 import workloads as W
from dcu_b200.api import Context, DcuError

pytestmark = pytest.mark.gpu


def _dev(A, b):
    import torch

    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return d(A.ptr), d(A.idx), d(A.val), d(b)


def test_autotune_reports_and_keeps_its_choice():
    A = W.convdiff3d(48, 20.0)
    b, _ = W.rhs_from_solution(A, seed=3)
    ptr, idx, val, bd = _dev(A, b)
    with Context(0) as c:
        t = c.autotune_d(A.n, A.nnz, ptr, idx, val, bd, reps=5, precision=N.PREC_M_BF16)
        # three kernels at >= 2 grids each, the fused step too (FP64 vectors), one build
        assert t.candidates >= 8, t.as_dict()
        assert t.k1_split in (0, 1)
        assert 0 < t.iter_us_tuned <= t.iter_us_default
        assert t.build_ms_default > 0 and t.build_ms_tuned <= t.build_ms_default
        # interior columns have |I| = 25: no lower limit would leave them on the warp kernel
        assert t.group_max_ni == 0
        for g in (t.grid_p, t.grid_y, t.grid_py, t.grid_sz):
            assert -1 <= g <= 64
        kept = c.get_tuning(N.PREC_M_BF16)
        assert all(getattr(kept, k) == getattr(t, k) for k in N.Tuning.CONFIG)
        assert c.get_tuning(N.PREC_FP64).k1_split == -1  # other forms untouched
        # a solve with the tuned configuration converges as the default one does
        x, _, _, si = c.solve_h(A, b, precision=N.PREC_M_BF16)
        assert si.status == N.SOLVE_CONVERGED
        assert np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b) < 1e-8


CONFIGS = [
    dict(k1_split=0), dict(k1_split=1),
    dict(grid_p=-1, grid_y=-1, grid_py=-1, grid_sz=-1),
    dict(grid_p=1, grid_y=2, grid_py=3, grid_sz=1),
    dict(k1_split=1, grid_p=4, grid_y=-1, grid_sz=2),
]


@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_M_BF16, N.PREC_M_FP32, N.PREC_MIXED_FP32])
def test_iteration_settings_leave_the_solution_bit_identical(prec):
    A = W.convdiff3d(20, 20.0)
    b, _ = W.rhs_from_solution(A, seed=5)
    with Context(0) as c:
        x0, m0, _, s0 = c.solve_h(A, b, want_m=True, precision=prec)
        assert s0.status == N.SOLVE_CONVERGED
        for cfg in CONFIGS:
            c.set_tuning(prec, **cfg)
            x, m, _, si = c.solve_h(A, b, want_m=True, precision=prec)
            assert si.iters == s0.iters and si.status == s0.status, cfg
            assert np.array_equal(m, m0), cfg
            assert np.array_equal(x, x0), cfg
        c.set_tuning(prec)  # back to the defaults
        x, _, _, si = c.solve_h(A, b, precision=prec)
        assert np.array_equal(x, x0)


def test_group_limit_moves_columns_to_the_cta_kernel():
    A = W.convdiff2d(64, 10.0)  # |I_k| <= 13
    b = W.rhs_ones_product(A)
    with Context(0) as c:
        m0, _, b0 = c.build_h(A)
        x0, _, _, s0 = c.solve_h(A, b)
        c.set_tuning(N.PREC_FP64, group_max_ni=8)
        m1, _, b1 = c.build_h(A)
        x1, _, _, s1 = c.solve_h(A, b)
    assert b0.cols_large == 0 and b1.cols_large > A.n // 2
    assert b1.cols_small + b1.cols_large == A.n
    # same pattern (A's), values equal up to rounding of a different reduction order
    assert np.max(np.abs(m1 - m0)) <= 1e-12 * np.max(np.abs(m0))
    assert abs(s1.iters - s0.iters) <= 1 and s1.status == N.SOLVE_CONVERGED


def test_out_of_range_settings_are_refused(ctx):
    for bad in (dict(k1_split=2), dict(grid_p=-2), dict(grid_sz=65), dict(group_max_ni=33)):
        with pytest.raises(DcuError):
            ctx.set_tuning(N.PREC_FP64, **bad)
    with pytest.raises(DcuError):
        ctx.set_tuning(7, k1_split=0)
    assert ctx.get_tuning(N.PREC_FP64).k1_split == -1
