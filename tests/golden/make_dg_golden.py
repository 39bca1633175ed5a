"""Writes tests/golden/dg_experiments.json from the reference's published results.

Run with DDX_REFERENCE_ROOT set to a checkout of the reference:
    DDX_REFERENCE_ROOT=<reference checkout>  python tests/golden/make_dg_golden.py

The reference logged every CG run of its DG-SIPG experiments, with the full
residual history, in ``results/experiment_precisions.csv`` and
``results/experiment_parallelism.csv`` (written by
``experiments/precision_experiments.py`` and
``experiments/parallelism_experiments.py`` through
``src/experiments/experiments/experiments.py:175-300``, on an A100). This
script keeps, for the 2D rows (continuous coefficient test case, uniform mesh
family, polynomial degrees 1, 3 and 5):

* ``p``                              - polynomial degree of the DG space,
* ``fine``, ``solvers``, ``coarse``  - mesh ids (``S<m>`` / ``C<m>``),
* ``solver``                         - the reference's ``str(solver)``,
* ``dofs``, ``nnz``                  - system size and matrix nnz,
* ``iterations``                     - CG iterations (``None`` if it failed),
* ``residual_norms``                 - the logged history (converged precision rows),
* ``solve_ms_min``                   - min over the logged solve times (ms).
"""
from __future__ import annotations

import ast
import csv
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("DDX_REFERENCE_ROOT")
if not REF:
    raise SystemExit("set DDX_REFERENCE_ROOT to a checkout of the reference (mgr0dzicki/dd-solvers)")

csv.field_size_limit(sys.maxsize)


def rows(name, keep_norms):
    out = []
    with open(os.path.join(REF, "results", name)) as fh:
        for r in csv.DictReader(fh):
            if not r["solver"].startswith("CG(") or r["p"] not in ("1", "3", "5"):
                continue
            md = r["metadata"]
            it = norms = None
            if md.startswith("{'iterations'"):
                meta = ast.literal_eval(md)
                it = meta["iterations"]
                # converged runs only: the failed ones ran to maxiter
                norms = meta["residual norms"] if keep_norms and it < 500 else None
            times = ast.literal_eval(r["solve times"]) if r["solve times"].startswith("[") else []
            out.append({
                "source": name,
                "test_case": r["test case"],
                "p": int(r["p"]),
                "fine": r["fine m"], "solvers": r["solvers m"], "coarse": r["coarse m"],
                "solver": r["solver"],
                "dofs": int(r["DoFs"]), "nnz": int(r["matrix nnz"]),
                "iterations": it,
                "residual_norms": norms,
                "solve_ms_min": min(times) if times else None,
                "exception": r["exception"] or None,
            })
    return out


def main():
    data = rows("experiment_precisions.csv", True) + rows("experiment_parallelism.csv", False)
    with open(os.path.join(HERE, "dg_experiments.json"), "w") as fh:
        json.dump(data, fh, separators=(",", ":"))
    print(len(data), "rows")


if __name__ == "__main__":
    main()
