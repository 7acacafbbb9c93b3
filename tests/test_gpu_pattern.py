"""Pattern kernel (J_k, I_k) against the oracle: bit-exact |I_k| and I_k."""
import numpy as np
import pytest

import oracle
from dcu_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _dev(A):
    import torch

    return (torch.from_numpy(np.ascontiguousarray(A.ptr)).cuda(), torch.from_numpy(np.ascontiguousarray(A.idx)).cuda())


def random_csc(n, density, seed, shuffle_rows=True, empty_cols=0):
    rng = np.random.Generator(np.random.PCG64(seed))
    cols = []
    for c in range(n):
        k = rng.binomial(n, density)
        rows = rng.choice(n, k, replace=False) if k else np.zeros(0, np.int64)
        if not shuffle_rows:
            rows = np.sort(rows)
        cols.append(rows)
    for c in rng.choice(n, empty_cols, replace=False):
        cols[c] = np.zeros(0, np.int64)
    ptr = np.zeros(n + 1, np.int64)
    ptr[1:] = np.cumsum([len(r) for r in cols])
    idx = np.concatenate(cols).astype(np.int32) if ptr[-1] else np.zeros(0, np.int32)
    val = rng.standard_normal(len(idx))
    return W.CSC(n, ptr.astype(np.int32), idx, val)


CASES = {
    "cd2d_64": lambda: W.convdiff2d(64, 10.0),
    "cd3d_12": lambda: W.convdiff3d(12, 20.0),
    "circuit": lambda: W.circuit_like(),
    "rand_unsorted": lambda: random_csc(700, 0.01, 1),
    "rand_dense_cols": lambda: random_csc(300, 0.08, 2, empty_cols=5),
    "varcoef_32": lambda: W.varcoef2d(32, seed=3),
}


@pytest.mark.parametrize("name", list(CASES))
def test_pattern_bit_exact(ctx, name):
    A = CASES[name]()
    cnt_o, iptr_o, il_o = oracle.pattern(A)
    p, i = _dev(A)
    cnt, iptr, il = ctx.pattern_d(A.n, p, i)
    assert np.array_equal(cnt.cpu().numpy(), cnt_o)
    assert np.array_equal(iptr.cpu().numpy(), iptr_o)
    assert np.array_equal(il.cpu().numpy(), il_o)


def test_pattern_column_range(ctx):
    A = W.circuit_like()
    s, e = 1000, 3217
    cnt_o, iptr_o, il_o = oracle.pattern(A, s, e)
    p, i = _dev(A)
    cnt, iptr, il = ctx.pattern_d(A.n, p, i, s, e)
    assert np.array_equal(cnt.cpu().numpy(), cnt_o)
    assert np.array_equal(il.cpu().numpy(), il_o)
