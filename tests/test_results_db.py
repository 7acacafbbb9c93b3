"""Results database: [ALGO_REPORT] / [SOLVER_REPORT] parsing, rows, the
reference's report format (CPU only)."""
import sqlite3

import pytest

from dcu_b200 import results_db as R

LOG = """matrix cd2d.mtx: n = 4096, nnz = 20224
[ALGO_REPORT] mode=static, dcu_units=1, partition=balanced_columns, preconditioner_ms=0.1234, iteration_count=43
[SOLVER_REPORT] gpupbicgstab_ms=0.9876, converged=1, solver_tol=1.000e-07, max_iters=10000
[ALGO_REPORT] mode=dynamic, dcu_units=1, partition=balanced_nnz, preconditioner_ms=0.2000, iteration_count=0
"""


def test_parse_pairs_solver_line_with_its_report():
    reps = R.parse_reports(LOG)
    assert len(reps) == 2
    a, b = reps
    assert (a.mode, a.dcu_units, a.partition, a.iteration_count) == ("static", 1, "balanced_columns", 43)
    assert a.preconditioner_ms == pytest.approx(0.1234) and a.gpupbicgstab_ms == pytest.approx(0.9876)
    assert a.converged == 1 and a.solver_tol == pytest.approx(1e-7) and a.max_iters == 10000
    # precondition-only run: no solver line of its own
    assert (b.mode, b.iteration_count, b.gpupbicgstab_ms, b.converged) == ("dynamic", 0, 0.0, 0)


def test_rows_and_report(tmp_path):
    db = str(tmp_path / "runs.sqlite")
    with R.connect(db) as conn:
        for rep in R.parse_reports(LOG):
            R.insert(conn, f"t-{rep.mode}", "cd2d", 4096, 20224, rep)
    with R.connect(db) as conn:   # re-opening keeps the rows and the two algorithms
        assert conn.execute("SELECT COUNT(*) FROM algorithms").fetchone()[0] == 2
        run = conn.execute("SELECT * FROM experiment_runs WHERE run_tag = 't-static'").fetchone()
        assert run["total_ms"] == pytest.approx(0.1234 + 0.9876)
        assert (run["matrix_rows"], run["matrix_nnz"], run["dcu_mode"], run["total_iters"]) == (4096, 20224,
                                                                                                 "single_gpu_cuda", 43)
        lines = R.report_lines(conn)
    assert lines[1] == ("t-static | cards=1 | static_spai_mpi | pre=0.12 ms | solver=0.99 ms | total=1.11 ms | "
                        "iters=43 | conv=1")
    assert lines[0].startswith("t-dynamic | cards=1 | dynamic_spai_mpi | pre=0.20 ms")


def test_checks_still_reject_bad_rows(tmp_path):
    with R.connect(str(tmp_path / "r.sqlite")) as conn:
        rep = R.parse_reports(LOG)[0]
        with pytest.raises(sqlite3.IntegrityError):
            R.insert(conn, "bad", "m", 1, 1, rep, dcu_mode="laptop")
        rep.converged = 2
        with pytest.raises(sqlite3.IntegrityError):
            R.insert(conn, "bad", "m", 1, 1, rep)


def test_ingest_and_report_cli(tmp_path, capsys):
    log = tmp_path / "run.log"
    log.write_text(LOG)
    db = str(tmp_path / "db" / "runs.sqlite")
    assert R.main(["report", "--db", db]) == 0
    assert "No benchmark records." in capsys.readouterr().out
    assert R.main(["ingest", "--db", db, "--log", str(log), "--matrix-name", "cd2d", "--rows", "4096",
                   "--nnz", "20224", "--tag", "night"]) == 0
    assert R.main(["report", "--db", db]) == 0
    out = capsys.readouterr().out.splitlines()
    assert [l.split(" | ")[0] for l in out] == ["night-dynamic", "night-static"]
    empty = tmp_path / "empty.log"
    empty.write_text("nothing here\n")
    assert R.main(["ingest", "--db", db, "--log", str(empty), "--matrix-name", "x", "--rows", "1",
                   "--nnz", "1"]) == 1
