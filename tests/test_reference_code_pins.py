"""The oracle against the reference's own code, run on the host
(oracle/_ref/libref_emu.so, built from the reference tree by `make emu`;
skipped where it was not built):

* SPAI: the reference's kernels (src/spai_single_dcu.cpp: computeJ*,
  computeI*, ComputeTildeACSR, QR_RShared (MGS), ComputeTildeE*, Sol,
  modifyData*) on the host SIMT emulator, with the reference's launch
  shapes, single-pass and tiled, against the oracle's MGS restatement.  They
  differ only where the reference's arithmetic is contracted into FMA (as
  HIP compiles device code): 1e-13 relative is a rounding-level bound.
* BiCGSTAB: the reference's cublas2_pbicgstabv2 (bicgstab_solver.h),
  compiled unmodified over host stand-ins of hipBLAS/hipSPARSE that sum as
  the oracle does, against the oracle's restatement on the same M: the same
  iteration count and bit-identical iterates, in the reference's solver
  settings and in the configs' (x0 = 0, threshold 1e-8 ||b||).
"""
import numpy as np
import pytest

import oracle
from dcu_b200 import api
from dcu_b200 import workloads as W
from tests.conftest import reference_file
from tests.test_gpu_pattern import random_csc

pytestmark = pytest.mark.skipif(not oracle.emu_available(), reason="reference kernels not built (no reference tree)")

CASES = {
    "convdiff2d_64": lambda: W.convdiff2d(64, 10.0),
    "convdiff3d_16": lambda: W.convdiff3d(16, 20.0),
    "varcoef2d_32": lambda: W.varcoef2d(32, seed=3),
    "circuit_like": lambda: W.circuit_like(),
    "rand_unsorted": lambda: random_csc(700, 0.01, 1),
    "fill_3elt.mtx": lambda: api.mtx_read(reference_file("matrices/fill_3elt.mtx")),
}


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", list(CASES))
def test_reference_kernels_match_oracle_mgs(name):
    A = CASES[name]()
    m_ref, info = oracle.refemu_spai(A)
    m_o, _, _, sing = oracle.spai(A, "mgs")
    assert np.isfinite(m_ref).all() and sing == 0
    assert _rel(m_ref, m_o) < 1e-13


def test_reference_tiled_path_is_exercised():
    # circuit-like: n * n1max * n2max exceeds the reference's single-pass size
    m_ref, (n1max, n2max, tiles, single) = oracle.refemu_spai(W.circuit_like())
    assert single == 0 and tiles > 1 and n2max > 256


@pytest.mark.parametrize("name", ["convdiff2d_64", "circuit_like", "convdiff3d_16"])
def test_reference_bicgstab_recurrence_matches_oracle(name):
    A = CASES[name]()
    m, _, _, _ = oracle.spai(A, "mgs")
    one = np.ones(A.n)
    r = oracle.refemu_bicgstab(A, m, one, one, 1e-7, 10000)
    o = oracle.bicgstab(A, m, one, one, tol=1e-7, tol_mode="abs", maxiter=10000)
    assert r["iters"] == o["iters"] and np.array_equal(r["x"], o["x"])
    b = W.rhs_ones_product(A)
    r = oracle.refemu_bicgstab(A, m, b, np.zeros(A.n), 1e-8 * np.linalg.norm(b), 1000)
    o = oracle.bicgstab(A, m, b, None, tol=1e-8, tol_mode="rel", maxiter=1000)
    assert r["iters"] == o["iters"] and np.array_equal(r["x"], o["x"])
