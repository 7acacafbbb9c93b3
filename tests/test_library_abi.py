"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute calls: this runs without a GPU)."""
import os
import re
import subprocess

import numpy as np
import pytest

from dcu_b200 import native as N
from dcu_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _exported():
    out = subprocess.run(["nm", "-D", "--defined-only", "-C", N.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    return out


def test_c_abi_symbols_exported():
    hdr = open(os.path.join(ROOT, "include", "dcu_spai.h")).read()
    names = set(re.findall(r"^\s*(?:int|void|const char\*|long long)\s+\**(dcu_\w+)\s*\(", hdr, re.M))
    assert len(names) >= 18
    exported = _exported()
    for n in names:
        assert re.search(rf"\b{n}\b", exported), n
    # the ctypes table covers the same set
    assert names == set(N.SIGNATURES)


def test_cpp_dropin_symbols_exported():
    hdr = open(os.path.join(ROOT, "include", "common", "spai_multi_dcu_api.h")).read()
    names = set(re.findall(r"^\s*(?:MultiDCU_Context\*|void|float|int|CSC_Matrix\*|const char\*)\s+(\w+)\(", hdr,
                           re.M))
    assert {"initMultiDCU", "cleanupMultiDCU", "RunStaticSPAI_MultiDCU_MPI", "RunDynamicSPAI_MultiDCU_MPI",
            "runBiCGSTABOnRank0"} <= names
    exported = _exported()
    for n in names:
        assert re.search(rf"\b{n}\(", exported), n


def test_library_loads_and_reports_no_device_cleanly():
    import ctypes as C

    L = N.lib()
    h = C.c_void_p()
    import torch

    rc = L.dcu_spai_create(C.byref(h), 0, 0)
    if torch.cuda.is_available():
        assert rc == N.OK
        L.dcu_spai_destroy(h)
    else:
        assert rc == N.ERR_NO_DEVICE and not h.value


def test_default_options():
    o = N.default_options()
    assert (o.schedule, o.precision, o.tol_mode, o.maxiter, o.tol, o.verify) == (0, 0, 1, 1000, 1e-8, 1)


@pytest.mark.parametrize("units", [1, 3, 7, 64])
@pytest.mark.parametrize("sched", [N.SCHED_BALANCED_COLUMNS, N.SCHED_BALANCED_NNZ])
def test_distribute_columns_matches_oracle(units, sched):
    import oracle
    from dcu_b200 import workloads as W

    A = W.circuit_like()
    for s, e in [(0, A.n), (17, 3001)]:
        s1, e1 = api.distribute_columns(A.ptr, s, e, units, sched)
        s2, e2 = oracle.distribute_columns(A.ptr, s, e, units, sched == N.SCHED_BALANCED_NNZ)
        assert np.array_equal(s1, s2) and np.array_equal(e1, e2)
        assert s1[0] == s and e1[-1] == e


def test_cli_help():
    out = subprocess.run([N.CLI_PATH, "--help"], capture_output=True, text=True)
    assert out.returncode == 0 and "--precondition-only" in out.stdout
