"""dcu_csc_to_csr_noalloc_d: the CSC -> CSR conversion for callers that cannot
allocate device memory (its scratch is a fixed array inside the library).

It is checked through the C ABI against dcu_csc_to_csr_d, the allocating
entry point, on two calls in a row with different matrices (the second call
finds the first call's leftovers in the shared scratch).  The conversion is
integer work plus a value gather, so the outputs must be identical.  This
file is named to run last; it passes alone and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from dcu_b200 import native as N
from dcu_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _convert_both(A):
    import torch

    from dcu_b200.api import Context

    L = N.lib()
    p, i, v = _dev(A.ptr), _dev(A.idx), _dev(A.val)
    outs = []
    for noalloc in (False, True):
        rp = torch.full((A.n + 1,), -7, dtype=torch.int32, device="cuda")
        ri = torch.full((max(1, A.nnz),), -7, dtype=torch.int32, device="cuda")
        rv = torch.full((max(1, A.nnz),), -7.0, dtype=torch.float64, device="cuda")
        if noalloc:
            stream = torch.cuda.current_stream().cuda_stream
            rc = L.dcu_csc_to_csr_noalloc_d(A.n, A.nnz, p.data_ptr(), i.data_ptr(), v.data_ptr(), rp.data_ptr(),
                                            ri.data_ptr(), rv.data_ptr(), C.c_void_p(stream))
            assert rc == N.OK, rc
        else:
            with Context(0) as ctx:
                ctx.csc_to_csr_d(A.n, A.nnz, p, i, v, rp, ri, rv)
        torch.cuda.synchronize()
        outs.append((rp.cpu().numpy(), ri.cpu().numpy(), rv.cpu().numpy()))
    return outs


def test_noalloc_matches_allocating_entry_point_twice():
    # first a skewed matrix with long rows (hub rows), then a stencil matrix
    for A in (W.circuit_like(), W.convdiff2d(64, 10.0)):
        (rp0, ri0, rv0), (rp1, ri1, rv1) = _convert_both(A)
        assert np.array_equal(rp0, rp1)
        assert np.array_equal(ri0, ri1)
        assert np.array_equal(rv0, rv1)


def test_noalloc_rejects_sizes_beyond_its_limit():
    L = N.lib()
    rc = L.dcu_csc_to_csr_noalloc_d(131073, 10, 1, 1, 1, 1, 1, 1, None)
    assert rc == N.ERR_LIMIT
    rc = L.dcu_csc_to_csr_noalloc_d(100, 1048577, 1, 1, 1, 1, 1, 1, None)
    assert rc == N.ERR_LIMIT


def _noalloc(A, ptr=None):
    """One dcu_csc_to_csr_noalloc_d call (optionally with a replaced ptr);
    returns (status, (rptr, ridx, rval))."""
    import torch

    L = N.lib()
    p = _dev(A.ptr if ptr is None else ptr)
    i, v = _dev(A.idx), _dev(A.val)
    rp = torch.zeros(A.n + 1, dtype=torch.int32, device="cuda")
    ri = torch.zeros(max(1, A.nnz), dtype=torch.int32, device="cuda")
    rv = torch.zeros(max(1, A.nnz), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.dcu_csc_to_csr_noalloc_d(A.n, A.nnz, p.data_ptr(), i.data_ptr(), v.data_ptr(), rp.data_ptr(),
                                    ri.data_ptr(), rv.data_ptr(), C.c_void_p(stream))
    torch.cuda.synchronize()
    return rc, (rp.cpu().numpy(), ri.cpu().numpy(), rv.cpu().numpy())


def _long_row_matrix(n=10000, row_len=9000):
    """A diagonal plus one row of row_len entries: n and nnz are inside the
    limits, the row is longer than the 8192 entries one row may hold."""
    cols = [[c] for c in range(n)]
    for c in range(1, row_len):
        cols[c].insert(0, 0)
    ptr = np.zeros(n + 1, np.int32)
    ptr[1:] = np.cumsum([len(c) for c in cols])
    idx = np.concatenate([np.array(c, np.int32) for c in cols])
    val = np.arange(1, len(idx) + 1, dtype=np.float64)
    return W.CSC(n, ptr, idx, val)


def test_noalloc_status_paths_leave_the_scratch_usable():
    """The statuses that depend on the shared scratch's flags: a row longer
    than 8192 entries (DCU_ERR_LIMIT, set inside the sort), then a malformed
    ptr (DCU_ERR_ARG, set by the input check); each time the next valid call
    returns DCU_OK with the allocating entry point's output, so the flags
    were cleared."""
    A = W.convdiff2d(64, 10.0)
    (rp0, ri0, rv0), _ = _convert_both(A)
    rc, _ = _noalloc(_long_row_matrix())
    assert rc == N.ERR_LIMIT
    rc, (rp, ri, rv) = _noalloc(A)
    assert rc == N.OK
    assert np.array_equal(rp, rp0) and np.array_equal(ri, ri0) and np.array_equal(rv, rv0)
    bad = A.ptr.copy()
    bad[5], bad[6] = bad[6], bad[5]             # ptr decreases
    rc, _ = _noalloc(A, bad)
    assert rc == N.ERR_ARG
    rc, (rp, ri, rv) = _noalloc(A)
    assert rc == N.OK
    assert np.array_equal(rp, rp0) and np.array_equal(ri, ri0) and np.array_equal(rv, rv0)


def test_noalloc_accepts_unsorted_columns():
    """Columns in any order (the input check's "unsorted" finding is not an
    error for the conversion): same output as the allocating entry point."""
    from tests.test_gpu_pattern import random_csc

    A = random_csc(2000, 0.004, 7)              # rows shuffled inside each column
    (rp0, ri0, rv0), (rp1, ri1, rv1) = _convert_both(A)
    assert np.array_equal(rp0, rp1) and np.array_equal(ri0, ri1) and np.array_equal(rv0, rv1)
