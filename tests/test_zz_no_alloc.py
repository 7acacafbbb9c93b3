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
