"""Regenerate tests/golden/golden.json from the CPU oracle (and, where the
reference tree is present, from the reference's own CPU helpers and its
MatrixMarket fixture).  Run: python tests/golden/make_golden.py"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from dcu_b200 import workloads as W  # noqa: E402

REF = "/root/reference"


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def case(name, A, b_kind):
    cnt, iptr, il = oracle.pattern(A)
    m, colres, E, sing = oracle.spai(A, "mgs")
    out = {"n": A.n, "nnz": A.nnz, "pattern_sha": digest(il), "icount_sha": digest(cnt), "max_ni": int(cnt.max()),
           "max_nj": int(np.diff(A.ptr).max()), "m_sum": float(m.sum()), "m_sumsq": float((m * m).sum()),
           "m_head": [float(v) for v in m[:8]], "colres_max": float(colres.max()), "singular": sing}
    ref = oracle.bicgstab(A, m, np.ones(A.n), np.ones(A.n), tol=1e-7, tol_mode="abs", maxiter=10000)
    out["iters_reference_settings"] = ref["iters"]
    if b_kind == "ones_product":
        b = W.rhs_ones_product(A)
    elif b_kind == "uniform":
        b = np.random.Generator(np.random.PCG64(11)).uniform(-1, 1, A.n)
    else:
        b = W.rhs_from_solution(A, seed=7)[0]
    cfg = oracle.bicgstab(A, m, b, None, tol=1e-8, tol_mode="rel", maxiter=1000)
    out["iters_config_settings"] = cfg["iters"]
    out["config_rel_res"] = cfg["true_res"] / float(np.linalg.norm(b))
    out["b"] = b_kind
    return out


def main():
    g = {
        "convdiff2d_64_pe10": case("cd2d", W.convdiff2d(64, 10.0), "ones_product"),
        "convdiff3d_16_pe20": case("cd3d", W.convdiff3d(16, 20.0), "solution"),
        "circuit_like_seed2024": case("circuit", W.circuit_like(), "uniform"),
    }
    path = os.path.join(REF, "matrices", "circuit_2.mtx")
    if os.path.exists(path) and oracle.ref_available():
        A = oracle.ref_mtx_read(path)
        cnt, _, il = oracle.pattern(A)
        g["circuit_2_mtx"] = {"n": A.n, "nnz": A.nnz, "ptr_sha": digest(A.ptr), "idx_sha": digest(A.idx),
                              "val_sha": digest(A.val), "n1max_reference": oracle.ref_n1max(A),
                              "n2max_reference": oracle.ref_n2max(A), "pattern_sha": digest(il)}
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json"), "w") as f:
        json.dump(g, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
