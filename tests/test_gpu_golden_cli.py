"""GPU results against the golden fixtures, and the command-line driver
(C++ drop-in API end to end) with its [ALGO_REPORT] line."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

from dcu_b200 import native as N
from dcu_b200 import workloads as W
from tests.test_golden import CASES, GOLDEN, digest, rhs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", list(CASES))
def test_gpu_matches_golden(ctx, name):
    import torch

    g = GOLDEN[name]
    A = CASES[name]()
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    cnt, _, il = ctx.pattern_d(A.n, d(A.ptr), d(A.idx))
    assert digest(il.cpu().numpy()) == g["pattern_sha"]
    m, res, info = ctx.build_h(A)
    assert abs(m.sum() - g["m_sum"]) <= 1e-10 * max(1.0, abs(g["m_sum"]))
    assert np.allclose(m[:8], g["m_head"], rtol=1e-10, atol=0)
    b = rhs(A, g["b"])
    x, _, bi, si = ctx.solve_h(A, b)
    assert si.status == N.SOLVE_CONVERGED
    assert abs(si.iters - g["iters_config_settings"]) <= 1


def write_mtx(path, A):
    cols = np.repeat(np.arange(A.n), np.diff(A.ptr))
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{A.n} {A.n} {A.nnz}\n")
        for r, c, v in zip(A.idx, cols, A.val):
            f.write(f"{r + 1} {c + 1} {v:.17g}\n")


@pytest.mark.parametrize("algo", ["static", "dynamic"])
def test_cli_algo_report(tmp_path, algo):
    A = W.convdiff2d(64, 10.0)
    path = tmp_path / "cd2d.mtx"
    write_mtx(str(path), A)
    out = subprocess.run([N.CLI_PATH, "--algo", algo, "--matrix", str(path)], capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0, out.stderr
    m = re.search(r"^\[ALGO_REPORT\] mode=(\w+), dcu_units=(\d+), partition=(\w+), preconditioner_ms=([0-9.]+), "
                  r"iteration_count=(\d+)$", out.stdout, re.M)
    assert m, out.stdout
    assert m.group(1) == algo
    assert m.group(3) == ("balanced_nnz" if algo == "dynamic" else "balanced_columns")
    assert abs(int(m.group(5)) - GOLDEN["convdiff2d_64_pe10"]["iters_reference_settings"]) <= 1
    out2 = subprocess.run([N.CLI_PATH, "--matrix", str(path), "--precondition-only"], capture_output=True,
                          text=True, timeout=120)
    assert out2.returncode == 0 and "iteration_count=0" in out2.stdout


def test_results_db_records_cli_runs(tmp_path):
    """`record` runs the driver (both partitions) and stores what it printed."""
    from dcu_b200 import results_db as R

    A = W.convdiff2d(64, 10.0)
    path = tmp_path / "cd2d.mtx"
    write_mtx(str(path), A)
    db = str(tmp_path / "runs.sqlite")
    assert R.main(["record", "--db", db, "--matrix", str(path), "--tag", "gpu"]) == 0
    with R.connect(db) as conn:
        rows = conn.execute("SELECT er.run_tag, er.matrix_rows, er.matrix_nnz, ram.iteration_count, ram.converged, "
                            "ram.preconditioner_ms, ram.gpupbicgstab_ms FROM run_algorithm_metrics ram "
                            "JOIN experiment_runs er ON er.id = ram.run_id ORDER BY er.run_tag").fetchall()
    assert [r["run_tag"] for r in rows] == ["gpu-dynamic", "gpu-static"]
    for r in rows:
        assert (r["matrix_rows"], r["matrix_nnz"]) == (A.n, A.nnz)
        assert abs(r["iteration_count"] - GOLDEN["convdiff2d_64_pe10"]["iters_reference_settings"]) <= 1
        assert r["converged"] == 1 and r["preconditioner_ms"] > 0 and r["gpupbicgstab_ms"] > 0
