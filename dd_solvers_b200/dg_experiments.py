"""The reference's own PCG experiments on its DG-SIPG problems, run through this package.

Counterpart of ``src/experiments/experiments/experiments.py:175-300`` (one CG
run: permute the system so that DOFs are grouped by (coarse cell, solver
cell), set up the solver with ``dofs_per_solver`` / ``solvers_per_coarse``,
time ``solve`` with CUDA events, min over repetitions, setup excluded) for the
configurations of ``experiments/precision_experiments.py`` and
``experiments/parallelism_experiments.py``: 2D, polynomial degree ``p`` = 1, 3
or 5 (``--degree``), continuous-coefficient test case, fine mesh ``S<m>``,
solver and coarse cells on ``S<k>`` triangles or ``C<k>`` quadrilaterals,
``CG(maxiter=2000, rtol=1e-9)``.

    python -m dd_solvers_b200.dg_experiments --fine S10 --solvers S8 --coarse S8 \\
        --method hybrid --precision f16
    python -m dd_solvers_b200.dg_experiments --degree 3 --fine S9 --solvers S8 --coarse S8
    python -m dd_solvers_b200.dg_experiments --all --log tests/golden/dg_experiments.json

(``--all``: every converged configuration the reference logged, one JSON line each.)

prints one JSON line per run: iterations, the min / median solve time over the
repetitions, and (when ``--log`` names the reference's logged results, e.g.
``tests/golden/dg_experiments.json``) the reference's iterations, its A100
solve time and the largest relative difference between the two residual
histories.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import dg
from .solvers import CG, CUDSS, AdditiveSchwarz, HybridSchwarz, Inv, asm_permutation, permute_csr_tensor

DT = {"f64": torch.float64, "f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}
REF_NAME = {torch.float64: "torch.float64", torch.float32: "torch.float32", torch.bfloat16: "torch.bfloat16",
            torch.float16: "torch.float16"}


def _quad_of(x, y, level):
    k = 1 << level
    ix = torch.clamp(torch.floor(x * k).to(torch.int64), 0, k - 1)
    iy = torch.clamp(torch.floor(y * k).to(torch.int64), 0, k - 1)
    return ix + iy * k


def solvers_to_coarse(solvers: str, coarse: str, device) -> torch.Tensor:
    """Solver cells to coarse cells, as ``UniformMeshes.get_mapping(solvers,
    coarse)`` (``meshing.py:238-261``): parents for S -> S, centroids for -> C."""
    ks, ls = solvers[0], int(solvers[1:])
    if ks == "S":
        mesh = dg.uniform_mesh_2d(ls, device)
        return dg.cell_mapping(mesh, coarse)
    if coarse[0] != "C":
        raise ValueError("quadrilateral solver cells need quadrilateral coarse cells")
    k = 1 << ls
    q = torch.arange(k * k, device=device)
    cx = ((q % k).to(torch.float64) + 0.5) / k
    cy = ((q // k).to(torch.float64) + 0.5) / k
    return _quad_of(cx, cy, int(coarse[1:]))


def build(fine: str, solvers: str, coarse: str, device="cuda", return_perm: bool = False, degree: int = 1):
    """Assemble ``S<fine>`` in the degree-p DG space and group its DOFs by
    (coarse, solver) as the reference does (``experiments.py:205-236``).
    Returns the permuted system and the setup keyword arguments (and, with
    ``return_perm``, the permutation: ``b_permuted = b[perm]``, so a solution
    maps back as ``x[inv(perm)]``)."""
    mesh = dg.uniform_mesh_2d(int(fine[1:]), device)
    system = dg.sipg(mesh, degree=degree)
    nb = system.block_size
    f2s = dg.cell_mapping(mesh, solvers)
    s2c = solvers_to_coarse(solvers, coarse, device)
    n_cells = mesh.n_cells
    f2d = torch.arange(nb * n_cells, device=device).view(n_cells, nb)
    perm = asm_permutation(f2s, s2c, f2d)
    inv = torch.empty_like(perm)
    inv[perm] = torch.arange(perm.numel(), device=device)
    load = system.load
    A = permute_csr_tensor(system.matrix, inv)
    del system
    b = load[perm]
    n_coarse = int(s2c.max()) + 1
    kwargs = dict(dofs_per_solver=int((f2s == 0).sum()) * nb,
                  solvers_per_coarse=torch.bincount(s2c, minlength=n_coarse),
                  block_size=nb)
    if return_perm:
        return A, b, kwargs, perm
    return A, b, kwargs


def reference_row(log, fine, solvers, coarse, method, pc_prec, block_prec, degree=1):
    if not log:
        return None
    name = "AdditiveSchwarz" if method == "additive" else "HybridSchwarz"
    inv = "Inv()" if block_prec == pc_prec else f"Inv({REF_NAME[block_prec]})"
    head = f"CG({name}({REF_NAME[pc_prec]}, {inv}, CUDSS"
    for r in log:
        if ((r["fine"], r["solvers"], r["coarse"]) == (fine, solvers, coarse) and r.get("p", 1) == degree
                and r["solver"].startswith(head)):
            return r
    return None


_NAME_DT = {"torch.float64": "f64", "torch.float32": "f32", "torch.bfloat16": "bf16", "torch.float16": "f16"}


def parse_solver(name: str) -> dict:
    """(method, preconditioner precision, block precision) of a logged
    ``str(CG(...))``, e.g. ``CG(HybridSchwarz(torch.float64,
    Inv(torch.float16), CUDSS), bsr_matmul=True)`` (the formats of
    ``solvers.py:209-210, 791-792, 844-845, 347-348``)."""
    head = "CG(AdditiveSchwarz(" if name.startswith("CG(AdditiveSchwarz(") else "CG(HybridSchwarz("
    if not name.startswith(head):
        raise ValueError(f"not a Schwarz-preconditioned CG: {name}")
    rest = name[len(head):]
    pc, rest = rest.split(", ", 1)
    if not rest.startswith("Inv("):
        raise ValueError(f"local solver is not Inv: {name}")
    blk = rest[len("Inv("):rest.index(")")]
    return {"method": "additive" if "Additive" in head else "hybrid", "pc_precision": _NAME_DT[pc],
            "precision": _NAME_DT[blk] if blk else _NAME_DT[pc]}


def logged_runs(log, degree=None, include_failed=False):
    """The converged runs of the reference's log (``make_dg_golden.py``
    rows), one per configuration, in log order; ``include_failed`` adds the
    ones that did not converge in 2000 iterations (they run to maxiter)."""
    seen, out = set(), []
    for r in log:
        if degree is not None and r.get("p", 1) != degree:
            continue
        if r["exception"] and (r["iterations"] is None or not include_failed):
            continue
        if r["iterations"] is None or (r["iterations"] >= 1999 and not include_failed):
            continue
        cfg = (r.get("p", 1), r["fine"], r["solvers"], r["coarse"], r["solver"])
        if cfg in seen:
            continue
        seen.add(cfg)
        out.append(dict(degree=cfg[0], fine=cfg[1], solvers=cfg[2], coarse=cfg[3], **parse_solver(r["solver"])))
    return out


def summarize(outs) -> dict:
    """Runs, how many reproduce the logged iteration count (exactly / within
    1), and the range of speed-ups against the logged A100 times."""
    ref = [o for o in outs if o.get("reference_iterations") is not None]
    sp = [o["reference_a100_solve_ms_min"] / o["solve_ms_min"] for o in ref if o.get("reference_a100_solve_ms_min")]
    return {"runs": len(outs), "with_reference": len(ref),
            "iterations_equal": sum(o["iterations"] == o["reference_iterations"] for o in ref),
            "iterations_within_1": sum(abs(o["iterations"] - o["reference_iterations"]) <= 1 for o in ref),
            "speedup_min": min(sp) if sp else None, "speedup_max": max(sp) if sp else None}


def run(fine, solvers, coarse, method, precision, pc_precision="f64", reps=10, log=None, flexible=False,
        device="cuda", degree=1) -> dict:
    t0 = time.perf_counter()
    A, b, kw = build(fine, solvers, coarse, device, degree=degree)
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t0
    pc_dt, blk_dt = DT[pc_precision], DT[precision]
    cls = HybridSchwarz if method == "hybrid" else AdditiveSchwarz
    cg = CG(cls(pc_dt, Inv(blk_dt) if blk_dt != pc_dt else Inv(), CUDSS()), rtol=1e-9, maxiter=2000,
            flexible=flexible)
    t0 = time.perf_counter()
    cg.setup(A, **kw)
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0
    x, meta = cg.solve(b)
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        x, meta = cg.solve(b)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    out = {"p": degree, "fine": fine, "solvers": solvers, "coarse": coarse, "method": method,
           "preconditioner_precision": pc_precision, "block_precision": precision,
           "flexible": bool(flexible), "dofs": int(A.shape[0]), "nnz": int(A.values().numel()),
           "dofs_per_solver": kw["dofs_per_solver"], "n_coarse": int(kw["solvers_per_coarse"].numel()),
           "iterations": meta["iterations"], "solve_ms_min": min(times),
           "solve_ms_median": float(np.median(times)), "setup_s": t_setup, "assembly_s": t_build,
           "residual_norms": meta["residual norms"]}
    ref = reference_row(log, fine, solvers, coarse, method, pc_dt, blk_dt, degree)
    if ref is not None:
        out["reference_iterations"] = ref["iterations"]
        out["reference_a100_solve_ms_min"] = ref["solve_ms_min"]
        if ref.get("residual_norms"):
            a = np.array(meta["residual norms"])
            r = np.array(ref["residual_norms"])
            k = min(len(a), len(r))
            out["history_max_rel_diff"] = float(np.max(np.abs(a[:k] - r[:k]) / np.abs(r[:k])))
            k10 = min(k, 10)
            out["history_max_rel_diff_first10"] = float(np.max(np.abs(a[:k10] - r[:k10]) / np.abs(r[:k10])))
    cg.destroy()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--degree", type=int, default=None, help="polynomial degree p of the DG space (default 1)")
    ap.add_argument("--fine", default="S10")
    ap.add_argument("--solvers", default="S8")
    ap.add_argument("--coarse", default="S8")
    ap.add_argument("--method", default="hybrid", choices=["additive", "hybrid"])
    ap.add_argument("--precision", default="f64", choices=list(DT), help="local block precision")
    ap.add_argument("--pc-precision", default="f64", choices=list(DT), help="preconditioner precision")
    ap.add_argument("--flexible", action="store_true", help="flexible (Polak-Ribiere) PCG")
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--log", default=None, help="JSON of the reference's logged runs")
    ap.add_argument("--history", action="store_true", help="print the residual history too")
    ap.add_argument("--all", action="store_true",
                    help="run every converged configuration of --log (restricted to --degree if given)")
    ap.add_argument("--include-failed", action="store_true",
                    help="with --all: also the configurations that did not converge for the reference")
    args = ap.parse_args()
    log = json.load(open(args.log)) if args.log else None
    if args.all:
        if log is None:
            ap.error("--all needs --log")
        outs = []
        for c in logged_runs(log, args.degree, args.include_failed):
            out = run(c["fine"], c["solvers"], c["coarse"], c["method"], c["precision"], c["pc_precision"],
                      args.reps, log, args.flexible, degree=c["degree"])
            if not args.history:
                out.pop("residual_norms")
            print(json.dumps(out), flush=True)
            outs.append(out)
            torch.cuda.empty_cache()
        print(json.dumps({"summary": summarize(outs)}), flush=True)
        return
    out = run(args.fine, args.solvers, args.coarse, args.method, args.precision, args.pc_precision,
              args.reps, log, args.flexible, degree=args.degree or 1)
    if not args.history:
        out.pop("residual_norms")
    print(json.dumps(out))


if __name__ == "__main__":
    main()
