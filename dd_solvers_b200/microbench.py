"""Kernel micro-benchmarks (counterparts of the reference's
experiments/benchmark_batched_gemv.py and experiments/benchmark_bsrmv.py).

    python -m dd_solvers_b200.microbench apply --n-el 64 --parts 8 --precision bf16 --rhs 1
    python -m dd_solvers_b200.microbench spmv --n-el 128 --rhs 1
    python -m dd_solvers_b200.microbench spmv --problem p1 --n-el 2048 --rhs 16
    python -m dd_solvers_b200.microbench bsr --n-el 2048 --p 1
    python -m dd_solvers_b200.microbench solve --workload c5 --precision f16
    python -m dd_solvers_b200.microbench gemv --ks 2,16,64,149

``apply`` times the Schwarz local-inverse apply (SIMT streaming kernel for
R < 16, tensor-core kernel for R in {16, 32, 64} with BF16/FP16 blocks) on the
3D Q1 box-partition problem; ``spmv`` times the FP64 SpMV. Each prints one
JSON line with the mean CUDA-event time per launch, the algorithmic bytes and
the achieved GB/s against the measured HBM peak.
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np
import torch

DT = {"f64": torch.float64, "f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}
ELT = {"f64": 8, "f32": 4, "bf16": 2, "f16": 2}


def _peak() -> float:
    p = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    return float(json.load(open(p))["hbm_gbs"]) if os.path.exists(p) else 6650.0


def _problem(n_el: int, parts: int, seed: int = 0):
    from . import partition, problems

    P = problems.diffusion3d_lognormal(n_el, seed)
    owner, nparts = partition.box_owner(P.interior_shape, parts)
    sub_ptr, sub_idx = partition.overlapping_subdomains(P.matrix, owner, nparts, 1)
    return P.matrix, sub_ptr, sub_idx, partition.q1_coarse_restriction(3, n_el, parts)


def _time(fn, reps: int, warm: int = 3) -> float:
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def bench_apply(args) -> dict:
    import dd_solvers_b200 as dd

    dev = torch.device("cuda")
    if args.problem == "p1":
        # jittered P1 mesh of n-el x n-el nodes, RCB into `parts` subdomains (the
        # C5 family; 724^2 nodes / 256 parts gives C5's block sizes, ~2200 DOFs)
        from . import partition, problems

        P = problems.p1_jittered(args.n_el, 0.3, 1.0, 0)
        owner = partition.rcb_owner(P.coords, args.parts)
        A = P.matrix
        sub_ptr, sub_idx = partition.overlapping_subdomains(A, owner, args.parts, 1)
    else:
        A, sub_ptr, sub_idx, R0 = _problem(args.n_el, args.parts)
    pc = dd.AdditiveSchwarz(torch.float64, dd.Inv(DT[args.precision]), None)
    pc.setup(dd.csr_to_torch(A).to(dev), subdomains=(sub_ptr, sub_idx))
    torch.cuda.empty_cache()  # release setup temporaries: a profiler then saves/restores less device memory
    R = args.rhs or 1
    pc.use_tensor_cores = not args.simt
    pc.rhs_terms = args.terms
    pc.tc_symmetric = not args.tc_full
    pc.autotune = args.tune
    pc.tc_stages = args.stages or None
    tune = None
    tc = pc._tc_ok(R) and pc.use_tensor_cores
    if args.tune and tc:
        pc.tune_tc(R)
        tune = {f"sym={sym},stages={st}": ms for (sym, st), ms in pc.tune_tc_timings[R].items()}
    elif args.tune:
        pc.tune(R)
        tune = {f"groups={g},stage_kb={kb}": ms for (g, kb), ms in pc.tune_timings.items()}
    r = torch.randn(A.shape[0] * R, dtype=torch.float64, device=dev)
    ms = _time(lambda: pc._local(r, R), args.reps)
    ks = pc.ks.astype(np.int64)
    n = A.shape[0]
    acc = 8 if pc.acc_dtype == torch.float64 else 4
    tc_cfg = pc._tc_config(R, pc._tc_terms(R)) if tc else (False, 0)
    tcsym = tc and tc_cfg[0]
    if tc:
        blk_bytes = pc._tile_store(True).nbytes if tcsym else int((ks * ks).sum() * ELT[args.precision])
    else:
        blk_bytes = pc.store.nbytes
    nbytes = int(blk_bytes + 4 * len(ks) + ks.sum() * 4 + n * R * 8 + ks.sum() * R * acc)
    kname = ("ddx_schwarz_local_apply_tc_sym" if tcsym else "ddx_schwarz_local_apply_tc") if tc else (
        "ddx_schwarz_local_apply_sym" if pc.store.layout == "sym" else "ddx_schwarz_local_apply")
    return {"kernel": kname, "precision": args.precision,
            "rhs": R, "rhs_terms": pc._tc_terms(R) if tc else None, "layout": pc.store.layout, "n_dofs": n, "subdomains": len(ks), "k_max": int(ks.max()), "ms_per_launch": ms,
            "algorithmic_bytes": nbytes, "achieved_gbs": nbytes / ms / 1e6, "frac_of_peak": nbytes / ms / 1e6 / _peak(),
            "tflops": 2.0 * float((ks * ks).sum()) * R / ms / 1e9,
            "config": ({"symmetric": tc_cfg[0], "stages": tc_cfg[1]} if tc else pc._apply_config(R)), "tune_ms": tune}


def bench_spmv(args) -> dict:
    import dd_solvers_b200 as dd
    from dd_solvers_b200 import _lib as L
    from .solvers import _SellMatrix

    from . import problems

    from . import partition

    dev = torch.device("cuda")
    if args.problem == "p1":
        P = problems.p1_jittered(args.n_el, 0.3, 1.0, 0)  # n_el = nodes per side
        owner = partition.rcb_owner(P.coords, args.parts) if args.order == "parts" else None
    elif args.problem == "q1_2d":
        P = problems.poisson2d(args.n_el)
    else:
        P = problems.diffusion3d_lognormal(args.n_el, 0)
    A = P.matrix
    if args.order == "parts":
        # DOFs numbered part by part (each part's DOFs keep their order): the
        # rows a CTA takes in turn then share most of their x rows
        if args.problem != "p1":
            owner, _ = partition.box_owner(P.interior_shape, args.parts)
        perm = np.argsort(owner, kind="stable")
        A = A[perm][:, perm].tocsr()
        A.sort_indices()
    M = _SellMatrix(dd.csr_to_torch(A).to(dev))
    if args.cluster >= 0:
        M.spmm_cluster = args.cluster
    R = args.rhs or 1
    x = torch.randn(A.shape[0] * R, dtype=torch.float64, device=dev)
    y = torch.empty_like(x)
    ms = _time(lambda: M.launch(x, y, R, L.SPMV_PLAIN), args.reps)
    n = A.shape[0]
    nbytes = A.nnz * 12 + (n + 1) * 4 + n * R * 16
    kern = "ddx_spmv_sell_f64" if R == 1 else ("ddx_spmv_csr_ordered_f64" if M._chunk_for(R) else "ddx_spmv_csr_f64")
    return {"kernel": kern, "problem": args.problem, "rhs": R, "cluster": M._chunk_for(R),
            "order": args.order,
            "n_dofs": n, "nnz": A.nnz, "ms_per_launch": ms, "algorithmic_bytes": nbytes,
            "achieved_gbs": nbytes / ms / 1e6, "frac_of_peak": nbytes / ms / 1e6 / _peak()}


def bench_bsr(args) -> dict:
    """BSR SpMV on the DG block structure of the reference's BSR benchmark
    (2D: the 2 n^2 triangles of an n x n grid; 3D: the 6 n^3 tetrahedra of an
    n^3 grid of cubes; P_p elements), FP64 values."""
    from dd_solvers_b200 import FastBSR, problems

    dev = torch.device("cuda")
    bs = problems.dg_block_size(args.dim, args.p)
    if args.dim == 2:
        crow, col = problems.dg_bsr_pattern_2d(args.n_el)
    else:
        crow, col = problems.dg_bsr_pattern_3d(args.n_el, device=dev)
    nbr, nnzb = len(crow) - 1, int(crow[-1])
    g = torch.Generator(device=dev).manual_seed(0)
    vals = torch.randn(nnzb, bs, bs, dtype=torch.float64, device=dev, generator=g)
    m = torch.sparse_bsr_tensor(torch.as_tensor(crow, device=dev), torch.as_tensor(col, device=dev), vals,
                                size=(nbr * bs, nbr * bs))
    A = FastBSR(m)
    del m, vals
    torch.cuda.empty_cache()
    x = torch.randn(nbr * bs, dtype=torch.float64, device=dev, generator=g)
    ms = _time(lambda: A @ x, args.reps)
    nbytes = nnzb * (bs * bs * 8 + 4) + (nbr + 1) * 4 + 2 * nbr * bs * 8
    return {"kernel": "ddx_spmv_bsr", "dim": args.dim, "p": args.p, "bs": bs, "dofs": nbr * bs, "bsr_nnz": nnzb,
            "ms_per_launch": ms, "algorithmic_bytes": nbytes, "achieved_gbs": nbytes / ms / 1e6,
            "frac_of_peak": nbytes / ms / 1e6 / _peak()}


def bench_gemv(args) -> dict:
    """The reference op ``gemv_strided_batched`` on its own benchmark's shapes
    (``experiments/benchmark_batched_gemv.py``): N = 2^27 // k^2 column-major
    k x k matrices with random entries, every (matrix, vector) dtype pair the
    op supports, for the k values of ``--ks``; CUDA-event time per launch."""
    from dd_solvers_b200 import gemv_strided_batched

    dev = torch.device("cuda")
    pairs = [("f32", "f32"), ("f16", "f32"), ("bf16", "f32"), ("f64", "f64"), ("f32", "f64"), ("f16", "f64"),
             ("bf16", "f64")]
    rows = []
    for k in [int(v) for v in args.ks.split(",")]:
        n = 2 ** 27 // (k * k)
        for a_dt, b_dt in pairs:
            g = torch.Generator(device=dev).manual_seed(k)
            A = torch.randn((n, k, k), device=dev, dtype=DT[a_dt], generator=g).transpose(1, 2).contiguous()
            A = A.transpose(1, 2)  # column-major, as the reference's benchmark builds it
            b = torch.randn((n, k), device=dev, dtype=DT[b_dt], generator=g)
            ms = _time(lambda: gemv_strided_batched(A, b, True), args.reps)
            nbytes = n * k * k * ELT[a_dt] + 2 * n * k * ELT[b_dt]
            rows.append({"k": k, "n": n, "A_dtype": a_dt, "b_dtype": b_dt, "ms": ms,
                         "achieved_gbs": nbytes / ms / 1e6, "frac_of_peak": nbytes / ms / 1e6 / _peak()})
            del A, b
    return {"kernel": "ddx_gemv_strided_batched", "rows": rows}


def bench_solve(args) -> dict:
    """One solve of a benchmark workload (``--workload``, block precision
    ``--precision``) inside a cudaProfilerStart/Stop window, after one warm-up
    solve: for launch lists (ncu --profile-from-start off)."""
    import dd_solvers_b200 as dd
    from dd_solvers_b200.workloads import WORKLOADS, build_problem, rhs_for

    spec = WORKLOADS[args.workload]
    prob = build_problem(spec)
    dev = torch.device("cuda")
    At = dd.csr_to_torch(prob["A"]).to(dev)
    cls = dd.HybridSchwarz if spec["method"] == "hybrid" else dd.AdditiveSchwarz
    cg = dd.CG(cls(torch.float64, dd.Inv(DT[args.precision]), dd.CUDSS()), rtol=2.5e-9, maxiter=2000,
               flexible=args.precision != "f64")
    cg.setup(At, subdomains=(prob["sub_ptr"], prob["sub_idx"]), coarse_restriction=prob["R0"], block_size=1)
    if args.restriction != "auto":
        cg.preconditioner.sub_restriction = args.restriction == "sub"
    cg.fuse_updates = args.fuse_updates == "on"
    if args.cluster >= 0:
        cg.matrix.spmm_cluster = args.cluster
    R = args.rhs or spec["R"]
    B = torch.as_tensor(rhs_for(prob["A"].shape[0], 0, 1, spec, R), device=dev)
    cg.solve(B)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.profiler.start()
    e0.record()
    _, meta = cg.solve(B)
    e1.record()
    torch.cuda.profiler.stop()
    torch.cuda.synchronize()
    its = meta["iterations"] if isinstance(meta["iterations"], int) else max(meta["iterations"])
    ms = e0.elapsed_time(e1)
    return {"workload": args.workload, "precision": args.precision, "rhs": R, "restriction": args.restriction,
            "fuse_updates": args.fuse_updates, "cluster": cg.matrix._chunk_for(R),
            "ms_per_solve": ms,
            "iterations": its, "ms_per_iteration": ms / max(its, 1)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["apply", "spmv", "bsr", "solve", "gemv"])
    ap.add_argument("--ks", default="2,4,8,16,24,32,48,64,100,128,149", help="gemv: block sizes")
    ap.add_argument("--workload", default="c5", help="solve: workload name (c1..c5)")
    ap.add_argument("--p", type=int, default=1, help="bsr: DG polynomial degree")
    ap.add_argument("--dim", type=int, default=2, choices=[2, 3], help="bsr: triangles (2) or tetrahedra (3)")
    ap.add_argument("--n-el", type=int, default=64)
    ap.add_argument("--problem", default="q1_3d", choices=["q1_3d", "p1", "q1_2d"],
                    help="spmv: 3D Q1 lognormal diffusion (n-el cells per side) or jittered P1 (n-el nodes per side)")
    ap.add_argument("--parts", type=int, default=8)
    ap.add_argument("--order", default="natural", choices=["natural", "parts"],
                    help="spmv: DOF numbering (natural grid order, or part by part with --parts)")
    ap.add_argument("--precision", default="bf16", choices=list(DT))
    ap.add_argument("--rhs", type=int, default=None, help="right-hand sides (apply/spmv: 1; solve: the workload's)")
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--simt", action="store_true", help="force the SIMT kernel for R >= 16")
    ap.add_argument("--tc-full", action="store_true", help="tensor-core apply on full blocks (not the upper triangle)")
    ap.add_argument("--terms", type=int, default=None, choices=[1, 2],
                    help="16-bit residual terms of the tensor-core apply (default: automatic)")
    ap.add_argument("--tune", action="store_true", help="run the autotuner first and report every candidate")
    ap.add_argument("--restriction", default="auto", choices=["auto", "sub", "y"],
                    help="solve: hybrid restriction for R >= 2 (per subdomain, or from y / the transpose map)")
    ap.add_argument("--cluster", type=int, default=-1,
                    help="spmv / solve, R >= 2: rows per breadth-first cluster of the SpMM work order (0: row order; "
                         "-1: the solver's default)")
    ap.add_argument("--fuse-updates", default="on", choices=["on", "off"],
                    help="solve: multi-RHS x update in the p update, unstored z (CG.fuse_updates)")
    ap.add_argument("--stages", type=int, default=0, help="apply: ring depth of the symmetric tensor-core kernel "
                                                          "(2..6; 0: deepest that fits)")
    args = ap.parse_args()
    out = {"apply": bench_apply, "spmv": bench_spmv, "bsr": bench_bsr, "solve": bench_solve,
           "gemv": bench_gemv}[args.what](args)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
