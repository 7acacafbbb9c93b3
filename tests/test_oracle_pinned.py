"""Pins against the reference's own CPU code, compiled from the reference tree
into oracle/_ref (skipped where that harness was not built: no reference tree):

* the library's MatrixMarket reader == readMatrixToCSC (read.h:1296-1320)
* the oracle's CSC->CSR == CSC2CSR (assemble.h:34-67)
* the oracle's max |I_k| / max |J_k| == computeN1MAX / computeN2MAX (init.h:43-92), and
  |I_k| of every column == computeN1MAX on a one-column M holding J_k
"""
import os

import numpy as np
import pytest

import oracle
from dcu_b200 import api
from dcu_b200 import workloads as W
from tests.conftest import reference_file

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="reference harness not built")

MTX_CASES = {
    "general_real": "%%MatrixMarket matrix coordinate real general\n% c\n3 3 5\n1 1 2.5\n3 1 -1\n2 2 4.0\n1 3 0.0\n3 3 7\n",
    "general_pattern": "%%MatrixMarket matrix coordinate pattern general\n3 3 4\n1 1\n2 1\n3 2\n2 3\n",
    "symmetric_real": "%%MatrixMarket matrix coordinate real symmetric\n%\n%\n4 4 5\n1 1 1.5\n2 1 -2\n3 2 0\n4 3 3.25\n4 4 9\n",
    "symmetric_pattern": "%%MatrixMarket matrix coordinate pattern symmetric\n3 3 3\n1 1\n3 1\n3 3\n",
    "unsorted_general": "%%MatrixMarket matrix coordinate real general\n4 4 6\n4 2 1\n1 2 2\n3 1 3\n1 1 4\n2 4 5\n4 4 6\n",
}


def _same(a, b):
    assert a.n == b.n and a.nnz == b.nnz
    assert np.array_equal(a.ptr, b.ptr)
    assert np.array_equal(a.idx, b.idx)
    assert np.array_equal(a.val, b.val)


@pytest.mark.parametrize("name", list(MTX_CASES))
def test_reader_small_cases(tmp_path, name):
    p = tmp_path / f"{name}.mtx"
    p.write_text(MTX_CASES[name])
    _same(api.mtx_read(str(p)), oracle.ref_mtx_read(str(p)))


@pytest.mark.parametrize("rel", ["matrices/circuit_2.mtx", "matrices/fill_3elt.mtx"])
def test_reader_fixtures(rel):
    path = reference_file(rel)
    _same(api.mtx_read(path), oracle.ref_mtx_read(path))


def _fixtures():
    out = [W.convdiff2d(32, 10.0), W.circuit_like(), W.varcoef2d(24, seed=1)]
    for name in ["circuit_2.mtx", "fill_3elt.mtx"]:
        p = oracle.fixture_path(name)
        if p is not None:
            out.append(api.mtx_read(p))
    return out


@pytest.mark.parametrize("k", range(5))
def test_csc2csr_pinned(k):
    mats = _fixtures()
    if k >= len(mats):
        pytest.skip("fixture absent")
    A = mats[k]
    a = oracle.csc2csr(A.n, A.ptr, A.idx, A.val)
    b = oracle.ref_csc2csr(A)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("k", range(5))
def test_sizing_pinned(k):
    mats = _fixtures()
    if k >= len(mats):
        pytest.skip("fixture absent")
    A = mats[k]
    cnt, _, _ = oracle.pattern(A)
    assert int(cnt.max()) == oracle.ref_n1max(A)
    assert int(np.diff(A.ptr).max()) == oracle.ref_n2max(A)


PER_COLUMN = {
    "convdiff2d_64": lambda: W.convdiff2d(64, 10.0),
    "circuit_like": lambda: W.circuit_like(),
    "varcoef2d_512": lambda: W.varcoef2d(512, seed=5),
    "convdiff3d_128": lambda: W.convdiff3d(128, 20.0),
    "circuit_2.mtx": lambda: api.mtx_read(reference_file("matrices/circuit_2.mtx")),
    "fill_3elt.mtx": lambda: api.mtx_read(reference_file("matrices/fill_3elt.mtx")),
}


@pytest.mark.parametrize("name", list(PER_COLUMN))
def test_every_column_sizing_pinned(name):
    """|I_k| of every column: the oracle's pattern pass == the reference's
    computeN1MAX run on a one-column M holding J_k (init.h:43-75)."""
    A = PER_COLUMN[name]()
    cnt, _, _ = oracle.pattern(A)
    assert np.array_equal(cnt, oracle.ref_n1_per_column(A))


def test_column_range_sizing_pinned():
    A = W.circuit_like()
    cnt, _, _ = oracle.pattern(A, 1000, 3217)
    assert np.array_equal(cnt, oracle.ref_n1_per_column(A, 1000, 3217))
