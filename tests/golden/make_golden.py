"""Regenerate tests/golden/golden.json from the CPU oracle (and, where the
reference tree is present, from the reference's own CPU helpers and its two
MatrixMarket fixtures).  Run: python tests/golden/make_golden.py
(the MGS build of circuit_2.mtx takes a few minutes); with --sensitivity it
writes tests/golden/sensitivity.json instead (see sensitivity()).

Per fixture it records the file's SHA-256 (the GPU tests check that the copy
they read is the reference's file), the reader's CSC digests, |I_k| of every
column from the reference's computeN1MAX, and the oracle's SPAI/BiCGSTAB
results in the reference's solver settings (b = 1, x0 = 1, ||r|| < 1e-7
absolute, MAX_ITER 10000) and in the configs' (b = A 1, x0 = 0, relative
1e-8, maxiter 1000)."""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from dcu_b200 import workloads as W  # noqa: E402



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


def file_sha256(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def fixture(path):
    A = oracle.ref_mtx_read(path)
    cnt, _, il = oracle.pattern(A)
    icount_ref = oracle.ref_n1_per_column(A)
    assert np.array_equal(cnt, icount_ref)
    m, colres, E, sing = oracle.spai(A, "mgs")
    out = {"file_sha256": file_sha256(path), "n": A.n, "nnz": A.nnz, "ptr_sha": digest(A.ptr),
           "idx_sha": digest(A.idx), "val_sha": digest(A.val), "icount_reference_sha": digest(icount_ref),
           "pattern_sha": digest(il), "max_ni": int(cnt.max()), "max_nj": int(np.diff(A.ptr).max()),
           "m_sum": float(m.sum()), "m_sumsq": float((m * m).sum()), "colres_max": float(colres.max()),
           "singular": sing, "diag_missing": int(A.n - sum(1 for k in range(A.n)
                                                           if k in A.idx[A.ptr[k]:A.ptr[k + 1]]))}
    r = oracle.bicgstab(A, m, np.ones(A.n), np.ones(A.n), tol=1e-7, tol_mode="abs", maxiter=10000)
    out["reference_settings"] = {"iters": r["iters"], "status": r["status"], "res": r["res"]}
    b = W.rhs_ones_product(A)
    r = oracle.bicgstab(A, m, b, None, tol=1e-8, tol_mode="rel", maxiter=1000)
    out["config_settings"] = {"iters": r["iters"], "status": r["status"],
                              "rel_res": r["true_res"] / float(np.linalg.norm(b))}
    if oracle.emu_available():
        # the same through the reference's own code: its SPAI kernels on the
        # host SIMT emulator, its BiCGSTAB over the host library stand-ins
        # (the config setting as its absolute threshold 1e-8 ||b|| with x0 = 0)
        me, info = oracle.refemu_spai(A)
        rr = oracle.refemu_bicgstab(A, me, np.ones(A.n), np.ones(A.n), 1e-7, 10000)
        rc = oracle.refemu_bicgstab(A, me, b, np.zeros(A.n), 1e-8 * float(np.linalg.norm(b)), 1000)
        out["reference_code"] = {
            "m_rel_diff_vs_oracle": float(np.max(np.abs(me - m)) / np.max(np.abs(m))),
            "single_pass": bool(info[3]), "tiles": int(info[2]), "n1max": int(info[0]), "n2max": int(info[1]),
            "reference_settings_iters": rr["iters"], "config_settings_iters": rc["iters"],
            "config_settings_rel_res": float(np.linalg.norm(b - A.matvec(rc["x"])) / np.linalg.norm(b))}
    return out


def main():
    g = {
        "convdiff2d_64_pe10": case("cd2d", W.convdiff2d(64, 10.0), "ones_product"),
        "convdiff3d_16_pe20": case("cd3d", W.convdiff3d(16, 20.0), "solution"),
        "circuit_like_seed2024": case("circuit", W.circuit_like(), "uniform"),
    }
    path = oracle.fixture_path("circuit_2.mtx")
    if path and oracle.ref_available():
        A = oracle.ref_mtx_read(path)
        cnt, _, il = oracle.pattern(A)
        g["circuit_2_mtx"] = {"n": A.n, "nnz": A.nnz, "ptr_sha": digest(A.ptr), "idx_sha": digest(A.idx),
                              "val_sha": digest(A.val), "n1max_reference": oracle.ref_n1max(A),
                              "n2max_reference": oracle.ref_n2max(A), "pattern_sha": digest(il)}
    fx = {}
    for name in ("circuit_2.mtx", "fill_3elt.mtx"):
        path = oracle.fixture_path(name)
        if path and oracle.ref_available():
            fx[name] = fixture(path)
    if fx:
        g["fixtures"] = fx
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json"), "w") as f:
        json.dump(g, f, indent=1, sort_keys=True)


def _perturbed(m, seed):
    """M with every value moved by one unit in the last place, up or down at
    random: a change below any summation-order difference."""
    s = np.random.Generator(np.random.PCG64(seed)).integers(0, 2, m.size).astype(bool)
    return np.where(s, np.nextafter(m, np.inf), np.nextafter(m, -np.inf))


def _block(A, s0, s1):
    sub_ptr = A.ptr[s0:s1 + 1] - A.ptr[s0]
    return W.CSC(s1 - s0, sub_ptr.astype(np.int32), (A.idx[A.ptr[s0]:A.ptr[s1]] - s0).astype(np.int32),
                 A.val[A.ptr[s0]:A.ptr[s1]])


def batch_sensitivity(trials=4, systems=64):
    """The same spread for every (system, right-hand side) pair of the first
    `systems` systems of the 512-system batch: the largest over the pairs."""
    bt = W.batch_systems()
    off = bt.offsets[: systems + 1].astype(np.int64)
    worst, moved = 0, 0
    for s in range(systems):
        As = _block(bt.A, int(off[s]), int(off[s + 1]))
        m, _, _, _ = oracle.spai(As, "mgs")
        mps = [_perturbed(m, t) for t in range(1, trials + 1)]
        for q in range(bt.B.shape[1]):
            b = bt.B[off[s]:off[s + 1], q]
            base = oracle.bicgstab(As, m, b, None, tol=1e-8, tol_mode="rel", maxiter=1000)["iters"]
            d = max(abs(oracle.bicgstab(As, mp, b, None, tol=1e-8, tol_mode="rel", maxiter=1000)["iters"] - base)
                    for mp in mps)
            worst = max(worst, d)
            moved += d > 0
    return {"iters_band": max(1, worst), "pairs": systems * bt.B.shape[1], "pairs_moved": moved,
            "trials": trials}


def fixture_sensitivity(trials=8):
    """The same spread on the reference's circuit_2 fixture, in the reference's
    solver settings and in the configs' (M from the Householder oracle)."""
    path = oracle.fixture_path("circuit_2.mtx")
    A = oracle.ref_mtx_read(path)
    m, _, _, _ = oracle.spai(A, "householder")
    one = np.ones(A.n)
    b = W.rhs_ones_product(A)
    runs = {"reference_settings": lambda mm: oracle.bicgstab(A, mm, one, one, tol=1e-7, tol_mode="abs",
                                                             maxiter=10000)["iters"],
            "config_settings": lambda mm: oracle.bicgstab(A, mm, b, None, tol=1e-8, tol_mode="rel",
                                                          maxiter=1000)["iters"]}
    out = {"trials": trials}
    for key, run in runs.items():
        base = run(m)
        its = [run(_perturbed(m, t)) for t in range(1, trials + 1)]
        out[key] = {"iters": base, "perturbed": its, "iters_band": max(1, max(abs(v - base) for v in its))}
    return out


def sensitivity(trials=8):
    """Spread of the oracle's own BiCGSTAB iteration count when M moves by one
    ulp per value, on the benchmark workloads with long solves: the band a
    solver with another summation order can be held to.  Writes
    tests/golden/sensitivity.json."""
    out = {"batch512_first64": batch_sensitivity()}
    A = W.varcoef2d(512, seed=5)
    rng = np.random.Generator(np.random.PCG64(5))
    b, xt = rng.standard_normal(A.n), rng.standard_normal(A.n)
    m, _, _, _ = oracle.spai(A, "mgs")
    base = oracle.bicgstab(A, m, b, None, tol=1e-8, tol_mode="rel", maxiter=3000)
    g = 2.0 * (base["x"] - xt)
    rp, ri, rv = oracle.csc2csr(A.n, A.ptr, A.idx, A.val)
    At = W.CSC(A.n, rp, ri, rv)
    fwd, adj = [], []
    base_t = oracle.bicgstab(At, oracle.csc2csr(A.n, A.ptr, A.idx, m)[2], g, None, tol=1e-8, tol_mode="rel",
                             maxiter=3000)
    for t in range(1, trials + 1):
        mp = _perturbed(m, t)
        fwd.append(oracle.bicgstab(A, mp, b, None, tol=1e-8, tol_mode="rel", maxiter=3000)["iters"])
        mt = oracle.csc2csr(A.n, A.ptr, A.idx, mp)[2]
        adj.append(oracle.bicgstab(At, mt, g, None, tol=1e-8, tol_mode="rel", maxiter=3000)["iters"])
    spread = lambda base_it, its: max(1, max(abs(v - base_it) for v in its))
    out["varcoef512"] = {"forward_iters": base["iters"], "forward_perturbed": fwd,
                         "forward_iters_band": spread(base["iters"], fwd),
                         "adjoint_iters": base_t["iters"], "adjoint_perturbed": adj,
                         "adjoint_iters_band": spread(base_t["iters"], adj), "trials": trials}
    A = W.convdiff3d(128, 20.0)
    b, _ = W.rhs_from_solution(A, seed=7)
    m, _, _, _ = oracle.spai(A, "mgs")
    base = oracle.bicgstab(A, m, b, None, tol=1e-8, tol_mode="rel", maxiter=1000)
    its = [oracle.bicgstab(A, _perturbed(m, t), b, None, tol=1e-8, tol_mode="rel", maxiter=1000)["iters"]
           for t in range(1, trials + 1)]
    out["convdiff3d_128"] = {"iters": base["iters"], "perturbed": its, "iters_band": spread(base["iters"], its),
                             "trials": trials}
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "sensitivity.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    if "--sensitivity" in sys.argv:
        sensitivity()
    elif "--fixture-sensitivity" in sys.argv:
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sensitivity.json")
        out = json.load(open(path))
        out["circuit_2_mtx"] = fixture_sensitivity()
        with open(path, "w") as f:
            json.dump(out, f, indent=1, sort_keys=True)
    elif "--batch-sensitivity" in sys.argv:
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sensitivity.json")
        out = json.load(open(path))
        out["batch512_first64"] = batch_sensitivity()
        with open(path, "w") as f:
            json.dump(out, f, indent=1, sort_keys=True)
    else:
        main()
