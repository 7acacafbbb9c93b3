"""Experiment results database: [ALGO_REPORT] runs recorded in SQLite.

The tables, column names and report query follow the reference's benchmark
database (experiments/schema.sql:5-52, experiments/benchmark_db.py:126-154),
so reports and ad-hoc queries written against it work on databases written
here.  Two things differ:

* the device columns admit a single CUDA GPU: ``dcu_mode`` also takes
  ``'single_gpu_cuda'`` and ``dcu_units`` / ``total_cards`` are any positive
  count (the reference's CHECKs allow only 1-3 DCUs of 2 cards each);
* rows come from real runs (the reference only inserts placeholder samples):
  ``record`` runs the command-line driver on a MatrixMarket file and parses
  its ``[ALGO_REPORT]`` line (preconditioner ms, iteration count) and its
  ``[SOLVER_REPORT]`` line (solver ms, converged, tolerance, iteration cap);
  ``ingest`` parses the same lines from a saved log.

A database created by the reference's schema keeps its own CHECKs; inserting
a single-GPU row into it fails with sqlite3.IntegrityError.

    python -m dcu_b200.results_db init   --db runs.sqlite
    python -m dcu_b200.results_db record --db runs.sqlite --matrix A.mtx [--algo static|dynamic|both] [--tag T]
    python -m dcu_b200.results_db ingest --db runs.sqlite --log run.log --matrix-name A --rows N --nnz Z [--tag T]
    python -m dcu_b200.results_db report --db runs.sqlite
"""
from __future__ import annotations

import argparse
import os
import re
import sqlite3
import subprocess
import sys
from dataclasses import dataclass

SCHEMA = """
PRAGMA foreign_keys = ON;

CREATE TABLE IF NOT EXISTS algorithms (
    id INTEGER PRIMARY KEY AUTOINCREMENT,
    name TEXT NOT NULL UNIQUE,
    class TEXT NOT NULL CHECK(class IN ('project_algo')),
    backend TEXT NOT NULL,
    partition_strategy TEXT NOT NULL CHECK(partition_strategy IN ('balanced_columns', 'balanced_nnz')),
    notes TEXT DEFAULT ''
);

CREATE TABLE IF NOT EXISTS experiment_runs (
    id INTEGER PRIMARY KEY AUTOINCREMENT,
    run_tag TEXT NOT NULL,
    matrix_name TEXT NOT NULL,
    matrix_rows INTEGER NOT NULL,
    matrix_cols INTEGER NOT NULL,
    matrix_nnz INTEGER NOT NULL,
    dcu_mode TEXT NOT NULL CHECK(dcu_mode IN ('single_node_multi_card', 'multi_node_multi_card_mpi_hip',
                                              'single_gpu_cuda')),
    dcu_units INTEGER NOT NULL CHECK(dcu_units >= 1),
    cards_per_dcu INTEGER NOT NULL DEFAULT 1 CHECK(cards_per_dcu >= 1),
    total_cards INTEGER NOT NULL CHECK(total_cards >= 1),
    node_count INTEGER NOT NULL,
    converged INTEGER NOT NULL CHECK(converged IN (0, 1)),
    solver_tol REAL NOT NULL,
    max_iters INTEGER NOT NULL,
    total_iters INTEGER NOT NULL,
    preconditioner_ms REAL NOT NULL,
    gpupbicgstab_ms REAL NOT NULL,
    total_ms REAL GENERATED ALWAYS AS (preconditioner_ms + gpupbicgstab_ms) STORED,
    created_at TEXT NOT NULL DEFAULT CURRENT_TIMESTAMP
);

CREATE TABLE IF NOT EXISTS run_algorithm_metrics (
    id INTEGER PRIMARY KEY AUTOINCREMENT,
    run_id INTEGER NOT NULL,
    algorithm_id INTEGER NOT NULL,
    preconditioner_ms REAL NOT NULL,
    gpupbicgstab_ms REAL NOT NULL,
    iteration_count INTEGER NOT NULL,
    converged INTEGER NOT NULL CHECK(converged IN (0, 1)),
    total_ms REAL GENERATED ALWAYS AS (preconditioner_ms + gpupbicgstab_ms) STORED,
    FOREIGN KEY(run_id) REFERENCES experiment_runs(id) ON DELETE CASCADE,
    FOREIGN KEY(algorithm_id) REFERENCES algorithms(id) ON DELETE CASCADE,
    UNIQUE(run_id, algorithm_id)
);

CREATE INDEX IF NOT EXISTS idx_runs_cards ON experiment_runs(dcu_mode, dcu_units, total_cards);
CREATE INDEX IF NOT EXISTS idx_runs_matrix ON experiment_runs(matrix_name);
CREATE INDEX IF NOT EXISTS idx_metrics_total ON run_algorithm_metrics(total_ms);

INSERT OR IGNORE INTO algorithms (name, class, backend, partition_strategy, notes) VALUES
    ('static_spai_mpi', 'project_algo', 'CUDA sm_100a', 'balanced_columns', 'RunStaticSPAI_MultiDCU_MPI'),
    ('dynamic_spai_mpi', 'project_algo', 'CUDA sm_100a', 'balanced_nnz', 'RunDynamicSPAI_MultiDCU_MPI');
"""

# experiments/benchmark_db.py:127-141, the reference's report
REPORT_QUERY = """
SELECT er.run_tag, er.total_cards, a.name AS algorithm, ram.preconditioner_ms, ram.gpupbicgstab_ms,
       ram.total_ms, ram.iteration_count, ram.converged
FROM run_algorithm_metrics ram
JOIN experiment_runs er ON er.id = ram.run_id
JOIN algorithms a ON a.id = ram.algorithm_id
ORDER BY er.total_cards ASC, a.name ASC;
"""

_ALGO = re.compile(r"^\[ALGO_REPORT\] mode=(\w+), dcu_units=(\d+), partition=(\w+), "
                   r"preconditioner_ms=([-0-9.eE+]+), iteration_count=(\d+)\s*$", re.M)
_SOLVER = re.compile(r"^\[SOLVER_REPORT\] gpupbicgstab_ms=([-0-9.eE+]+), converged=([01]), "
                     r"solver_tol=([-0-9.eE+]+), max_iters=(\d+)\s*$", re.M)


@dataclass
class Report:
    mode: str               # static | dynamic
    dcu_units: int
    partition: str          # balanced_columns | balanced_nnz
    preconditioner_ms: float
    iteration_count: int
    gpupbicgstab_ms: float = 0.0
    converged: int = 0
    solver_tol: float = 1e-7
    max_iters: int = 10000


def parse_reports(text: str) -> list[Report]:
    """Every [ALGO_REPORT] line of a run's output, each paired with the
    [SOLVER_REPORT] line that follows it before the next [ALGO_REPORT] (a
    --precondition-only run has none: solver time 0, not converged)."""
    out = []
    algos = list(_ALGO.finditer(text))
    for i, m in enumerate(algos):
        end = algos[i + 1].start() if i + 1 < len(algos) else len(text)
        r = Report(m.group(1), int(m.group(2)), m.group(3), float(m.group(4)), int(m.group(5)))
        s = _SOLVER.search(text, m.end(), end)
        if s:
            r.gpupbicgstab_ms, r.converged = float(s.group(1)), int(s.group(2))
            r.solver_tol, r.max_iters = float(s.group(3)), int(s.group(4))
        out.append(r)
    return out


def connect(path: str) -> sqlite3.Connection:
    conn = sqlite3.connect(path)
    conn.row_factory = sqlite3.Row
    conn.executescript(SCHEMA)
    return conn


def insert(conn: sqlite3.Connection, run_tag: str, matrix_name: str, rows: int, nnz: int, rep: Report,
           dcu_mode: str = "single_gpu_cuda", total_cards: int = 1, node_count: int = 1) -> int:
    """One experiment_runs row and its run_algorithm_metrics row; returns the run id."""
    algo = {"static": "static_spai_mpi", "dynamic": "dynamic_spai_mpi"}[rep.mode]
    algo_id = conn.execute("SELECT id FROM algorithms WHERE name = ?", (algo,)).fetchone()["id"]
    cur = conn.execute(
        "INSERT INTO experiment_runs (run_tag, matrix_name, matrix_rows, matrix_cols, matrix_nnz, dcu_mode, "
        "dcu_units, cards_per_dcu, total_cards, node_count, converged, solver_tol, max_iters, total_iters, "
        "preconditioner_ms, gpupbicgstab_ms) VALUES (?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?)",
        (run_tag, matrix_name, rows, rows, nnz, dcu_mode, rep.dcu_units, 1, total_cards, node_count, rep.converged,
         rep.solver_tol, rep.max_iters, rep.iteration_count, rep.preconditioner_ms, rep.gpupbicgstab_ms))
    run_id = cur.lastrowid
    conn.execute(
        "INSERT INTO run_algorithm_metrics (run_id, algorithm_id, preconditioner_ms, gpupbicgstab_ms, "
        "iteration_count, converged) VALUES (?, ?, ?, ?, ?, ?)",
        (run_id, algo_id, rep.preconditioner_ms, rep.gpupbicgstab_ms, rep.iteration_count, rep.converged))
    return run_id


def report_lines(conn: sqlite3.Connection) -> list[str]:
    """The reference's report format (experiments/benchmark_db.py:150-154)."""
    return [f"{r['run_tag']} | cards={r['total_cards']} | {r['algorithm']} | "
            f"pre={r['preconditioner_ms']:.2f} ms | solver={r['gpupbicgstab_ms']:.2f} ms | "
            f"total={r['total_ms']:.2f} ms | iters={r['iteration_count']} | conv={r['converged']}"
            for r in conn.execute(REPORT_QUERY).fetchall()]


def run_cli(matrix: str, algo: str, extra: list[str] | None = None, cli: str | None = None) -> str:
    """Run the command-line driver on a MatrixMarket file; its stdout."""
    from dcu_b200 import native

    cmd = [cli or native.CLI_PATH, "--algo", algo, "--matrix", matrix] + list(extra or [])
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"{' '.join(cmd)} failed ({out.returncode}): {out.stderr.strip()}")
    return out.stdout


def _matrix_size(text: str) -> tuple[int, int]:
    m = re.search(r"^matrix .*: n = (\d+), nnz = (\d+)$", text, re.M)
    if not m:
        raise ValueError("driver output has no 'matrix ...: n = N, nnz = Z' line")
    return int(m.group(1)), int(m.group(2))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m dcu_b200.results_db")
    ap.add_argument("action", choices=["init", "record", "ingest", "report"])
    ap.add_argument("--db", required=True)
    ap.add_argument("--matrix", help="MatrixMarket file (record)")
    ap.add_argument("--algo", default="both", choices=["static", "dynamic", "both"])
    ap.add_argument("--tag", default="run")
    ap.add_argument("--log", help="saved driver output (ingest)")
    ap.add_argument("--matrix-name")
    ap.add_argument("--rows", type=int)
    ap.add_argument("--nnz", type=int)
    a = ap.parse_args(argv)
    if os.path.dirname(a.db):
        os.makedirs(os.path.dirname(a.db), exist_ok=True)
    with connect(a.db) as conn:
        if a.action == "record":
            if not a.matrix:
                ap.error("record needs --matrix")
            name = os.path.splitext(os.path.basename(a.matrix))[0]
            for algo in (["static", "dynamic"] if a.algo == "both" else [a.algo]):
                text = run_cli(a.matrix, algo)
                rows, nnz = _matrix_size(text)
                for rep in parse_reports(text):
                    insert(conn, f"{a.tag}-{rep.mode}", name, rows, nnz, rep)
        elif a.action == "ingest":
            if not (a.log and a.matrix_name and a.rows and a.nnz is not None):
                ap.error("ingest needs --log, --matrix-name, --rows and --nnz")
            with open(a.log, encoding="utf-8") as f:
                reps = parse_reports(f.read())
            if not reps:
                print(f"no [ALGO_REPORT] line in {a.log}", file=sys.stderr)
                return 1
            for rep in reps:
                insert(conn, f"{a.tag}-{rep.mode}", a.matrix_name, a.rows, a.nnz, rep)
        elif a.action == "report":
            lines = report_lines(conn)
            print("\n".join(lines) if lines else "No benchmark records.")
    return 0


if __name__ == "__main__":
    sys.exit(main())
