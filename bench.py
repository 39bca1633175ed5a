"""Benchmark: time per right-hand side to 1e-8 relative error, mixed precision vs FP64.

Default workload (C2, the headline): 3D Q1 diffusion on 128^3 hexahedra
(127^3 = 2,048,383 DOFs), kappa = exp(g), g i.i.d. N(0,1) per element (seed 0);
16^3 = 4096 box subdomains with one layer of overlap; Q1 coarse space on the
subdomain vertices (15^3 = 3375 coarse DOFs); Hybrid Schwarz with local inverse
blocks stored in BF16 (per-block power-of-two scale, FP32 accumulation); FP64
flexible PCG. One step = one PCG solve of one right-hand side (uniform[-1,1],
seeded). The relative error of every timed solution against the FP64 reference
solution (the FP64 plain path at rtol 1e-12) is checked to be <= 1e-8; the
stopping tolerance is tightened until it is.

Other workloads (--workload): c1 2D Q1 Poisson 256^2, 8x8 subdomains, additive
Schwarz; c3 2D Q1 Poisson 1024^2, 32x32 subdomains, 64 right-hand sides per
solve on the tensor cores; c4 the gradient of ||u - u_t||^2 for 2D Q1 diffusion
on 512^2 cells with kappa = exp(Gaussian random field) (one step = forward
solve + adjoint solve + element-gradient kernel, checked against central
differences along 16 seeded directions); c5 jittered P1 on 2048^2 nodes, RCB
into 2048 uneven subdomains, 16 right-hand sides per solve (block terms from
--precision: BF16 uses two 16-bit residual terms, FP16 one). For several
right-hand sides a step is one solve of the whole block and the time is
divided by their number.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c2]

At N = 1 the c2 line also carries "reference_experiment": the reference's own DG-SIPG experiment S10 / S8 /
S8 (hybrid, FP16 blocks) solved through this package, next to the reference's logged A100 time for it (and
the same experiment at P3 on S9 and P5 on S8 under "higher_degree");
"multi_rhs": compact c3 and c5 results; "other_workloads": compact c1 and c4 results (short timing).

--impl reference times the FP64 CPU restatement of the same algorithm on the
host cores (the reference's own solver runs on GPUs only; its CPU behaviour is
what the restatement reproduces) on a bounded sample of the workload.

With --gpus N > 1 (torchrun), every rank solves its own right-hand sides on its
own replica of the problem (the path needs no exchange between GPUs: weak
scaling, no collective in the solve); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}

from dd_solvers_b200.workloads import WORKLOADS, build_problem, rhs_for  # noqa: E402


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]), "source": "measured"}
    return dict(PEAKS_FALLBACK, source="fallback")


class Clocks:
    """nvidia-smi sampler for the timed region (clocks and throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int, interval_ms: int = 200):
        self.idx = device_index
        self.interval_ms = interval_ms
        self.proc = None
        # raw samples go to DDX_CLOCKS_DIR (default: the system temp directory); the line carries the summary
        self.path = os.path.join(os.environ.get("DDX_CLOCKS_DIR", tempfile.gettempdir()),
                                 f"ddx_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.interval_ms)],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: FP64 restatement, bounded sample
# ---------------------------------------------------------------------------

def host_inverses(prob):
    """FP64 inverses of every local block on the host cores (setup of the CPU
    solve, not timed): one block per worker thread, one BLAS thread each."""
    from concurrent.futures import ThreadPoolExecutor

    from threadpoolctl import threadpool_limits

    from oracle import restatement as orc

    A, sp, si = prob["A"], prob["sub_ptr"], prob["sub_idx"]

    def inv(i):
        idx = si[sp[i]:sp[i + 1]]
        return np.linalg.inv(orc.local_block(A, idx)) if len(idx) else np.zeros((0, 0))

    with threadpool_limits(1):
        with ThreadPoolExecutor(os.cpu_count()) as ex:
            return list(ex.map(inv, range(len(sp) - 1)))


def cpu_solve_per_rhs(prob, spec, rtol, inverse_blocks, repeats: int = 1):
    """CPU baseline: full FP64 Schwarz-PCG solves of one right-hand side of the
    workload with the oracle restatement on the host cores, run the way the
    reference runs its solver on CPU tensors: the equal-size local blocks applied
    by one batched matrix product per size and the sparse products through
    torch's threaded CSR kernel, every host thread. Timed like the reference times
    its solves: the minimum over ``repeats`` solves, setup excluded (the FP64
    inverse blocks are given)."""
    import torch
    from threadpoolctl import threadpool_limits

    from oracle import restatement as orc

    torch.set_num_threads(os.cpu_count())
    from dd_solvers_b200.setup_ops import scipy_csr

    A, R0 = prob["A"], scipy_csr(prob["R0"])
    M = orc.Schwarz(A, prob["sub_ptr"], prob["sub_idx"], R0, inverse_blocks=inverse_blocks, batched=True)
    Ah = orc.HostCSR(A)
    n = A.shape[0]
    b = rhs_for(n, 0, 1, spec)
    b = b if b.ndim == 1 else b[:, 0]
    times, its = [], None
    # NumPy's BLAS pool kept to one thread: its spinning workers would otherwise
    # contend with torch's for the same cores (measured 10x slower solves)
    with threadpool_limits(1, user_api="blas"):
        for _ in range(max(1, repeats)):
            t0 = time.perf_counter()
            if spec["method"] == "hybrid":
                _, m = orc.pcg(Ah, b, M.hybrid, rtol=rtol, T0=M.T0, maxiter=5000)
            else:
                _, m = orc.pcg(Ah, b, M.additive, rtol=rtol, maxiter=5000)
            times.append(time.perf_counter() - t0)
            its = m["iterations"]
            if sum(times) > 60.0:  # a long CPU solve is timed once
                break
    return {"ms_per_rhs": min(times) * 1e3, "iterations": its, "cores": os.cpu_count(), "solves": len(times),
            "sample": (f"full FP64 {spec['method']} Schwarz-PCG solve of one right-hand side on the whole problem "
                       f"({n} DOFs, {len(prob['sub_ptr']) - 1} subdomains) with the oracle restatement to rtol "
                       f"{rtol:g} (local blocks by torch.bmm per block size, torch CSR products, "
                       f"{torch.get_num_threads()} threads), {its} iterations, min over {len(times)} solve(s), "
                       f"setup excluded")}


def gpu_blocks_to_host(pc):
    """The FP64 inverse blocks of a GPU Schwarz operator (symmetrised, as the
    solver applies them), copied to the host for the CPU baseline."""
    return [pc.store.block(i).cpu().numpy() for i in range(pc.n_solvers)]


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def run_grad(args, spec, rank: int, world: int):
    """c4: time per gradient of L = ||u(kappa, f) - u_t||^2 w.r.t. (kappa, f).

    One step = forward PCG solve + loss + backward (adjoint PCG solve, mass
    scaling, element-gradient kernel), FP64 vectors, local blocks of the head
    precision (FP64 for comparison). The gradient is checked against central
    differences (h = 1e-6) along 16 seeded directions in (kappa, f).
    """
    import torch
    import torch.distributed as dist

    import dd_solvers_b200 as dd
    from dd_solvers_b200 import _lib as L
    from dd_solvers_b200 import problems, replicas

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    prob = build_problem(spec)
    n_el = spec["n_el"]
    op = dd.Q1Diffusion(2, n_el, dev)
    n = op.n
    kappa = torch.as_tensor(np.exp(problems.gaussian_random_field(n_el, 0.1, seed=0)), device=dev)
    kappa_t = torch.as_tensor(np.exp(problems.gaussian_random_field(n_el, 0.1, seed=1)), device=dev)
    f = torch.ones(n, dtype=torch.float64, device=dev)
    head = args.precision
    dts = {"f64": torch.float64, "bf16": torch.bfloat16, "f32": torch.float32, "f16": torch.float16}
    t0 = time.time()
    cgs = {}
    for prec in ("f64", head):
        cg = dd.CG(dd.AdditiveSchwarz(torch.float64, dd.Inv(dts[prec]), dd.CUDSS()), rtol=1e-10, maxiter=5000,
                   check_every=args.check_every, flexible=(prec != "f64"))
        cg.setup(op.matrix(kappa), subdomains=(prob["sub_ptr"], prob["sub_idx"]), owner=prob["owner"],
                 block_size=1)
        cgs[prec] = cg
    torch.cuda.synchronize()
    gpu_setup_s = time.time() - t0
    with torch.no_grad():
        ut = dd.DiffusionSolve.apply(kappa_t, f, op, cgs["f64"])

    def grad_step(cg, k, ff):
        k = k.detach().requires_grad_(True)
        ff = ff.detach().requires_grad_(True)
        u = dd.DiffusionSolve.apply(k, ff, op, cg)
        loss = ((u - ut) ** 2).sum()
        loss.backward()
        return loss.detach(), k.grad, ff.grad

    def timed(prec, k_steps, w, host=False, count=False):
        cg = cgs[prec]
        if host:
            kh, fh = kappa.cpu().pin_memory(), f.cpu().pin_memory()
            gkh = torch.empty_like(kh).pin_memory()
            gfh = torch.empty_like(fh).pin_memory()
            lh = torch.empty((), dtype=torch.float64).pin_memory()
            kd, fd = torch.empty_like(kappa), torch.empty_like(f)
        for _ in range(w):
            grad_step(cg, kappa, f)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        if count:
            L.CALLS[0] = 0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k_steps):
            if host:
                kd.copy_(kh, non_blocking=True)
                fd.copy_(fh, non_blocking=True)
                loss, gk, gf = grad_step(cg, kd, fd)
                gkh.copy_(gk, non_blocking=True)
                gfh.copy_(gf, non_blocking=True)
                lh.copy_(loss, non_blocking=True)
            else:
                grad_step(cg, kappa, f)
        e1.record()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        return replicas.max_over_ranks(e0.elapsed_time(e1) / k_steps, dev)

    steps, warm = args.steps, args.warmup
    clocks = Clocks(dev.index if dev.index is not None else 0)
    clocks.start()
    ms_head = timed(head, steps, warm, count=True)
    clk = clocks.stop()
    launches = L.CALLS[0]
    ms_f64 = timed("f64", max(1, min(steps, 3)), 1)
    ms_e2e = timed(head, steps, 1, host=True)

    # gradient check: central differences along 16 seeded directions (tight solves)
    cgc = cgs[head]
    rtol_run = cgc.rtol
    cgc.rtol = 1e-12
    _, gk, gf = grad_step(cgc, kappa, f)
    rng = np.random.default_rng(123)
    h = 1e-6
    worst = 0.0
    with torch.no_grad():
        for _ in range(16):
            dk = torch.as_tensor(rng.standard_normal(kappa.shape), device=dev) * kappa
            df = torch.as_tensor(rng.standard_normal(n), device=dev)
            lp = float(((dd.DiffusionSolve.apply(kappa + h * dk, f + h * df, op, cgc) - ut) ** 2).sum())
            lm = float(((dd.DiffusionSolve.apply(kappa - h * dk, f - h * df, op, cgc) - ut) ** 2).sum())
            fd_ = (lp - lm) / (2 * h)
            ad = float((gk * dk).sum() + (gf * df).sum())
            worst = max(worst, abs(fd_ - ad) / max(abs(ad), 1e-30))
    cgc.rtol = rtol_run
    # gradient agreement between the head precision and FP64 blocks at the run tolerance
    _, gk64, gf64 = grad_step(cgs["f64"], kappa, f)
    _, gkh_, gfh_ = grad_step(cgs[head], kappa, f)
    grad_rel = float(torch.linalg.norm(gkh_ - gk64) / torch.linalg.norm(gk64))

    # dominant kernel: the element gradient + local apply are small here; report the local apply
    pc = cgs[head].preconditioner
    r = torch.randn(n, dtype=torch.float64, device=dev)
    for _ in range(3):
        pc._local(r, 1)
    kev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    kev[0].record()
    for _ in range(20):
        pc._local(r, 1)
    kev[1].record()
    torch.cuda.synchronize()
    k_ms = kev[0].elapsed_time(kev[1]) / 20
    ks = pc.ks.astype(np.int64)
    elt = {"f64": 8, "f32": 4, "bf16": 2, "f16": 2}[head]
    alg_bytes = int(pc.store.nbytes + 4 * len(ks) + ks.sum() * 4 + n * 8 + ks.sum() * 4)
    peaks = load_peaks()
    out = None
    if rank == 0:
        ach = alg_bytes / (k_ms * 1e-3) / 1e9
        out = {
            "metric": "time per gradient (forward + adjoint Schwarz PCG to rtol 1e-10 + element gradient), 1 B200",
            "value": ms_head / world, "unit": "ms/gradient", "n_gpus": world, "steps": steps, "warmup": warm,
            "ms_per_step": ms_head, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": f"{head} blocks / f64 PCG", "data": "synthetic (seeded Gaussian random fields)",
            "config": {"workload": f"{args.workload}: {spec['name']}, {head} blocks", "n_dofs": n,
                       "subdomains": prob["nparts"], "k_max": int(ks.max()),
                       "l2": "inputs smaller than L2; every step re-assembles A(kappa) and solves twice",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "fp64_blocks_ms_per_gradient": ms_f64, "speedup_vs_fp64_blocks": ms_f64 / ms_head,
            "gradient_check": {"directions": 16, "h": h, "max_rel_err_fd_vs_adjoint": worst,
                               "head_vs_fp64_blocks_grad_rel_diff": grad_rel},
            "e2e": {"value": ms_e2e / world, "unit": "ms/gradient", "h2d_bytes_per_step": (kappa.numel() + n) * 8,
                    "d2h_bytes_per_step": (kappa.numel() + n + 1) * 8},
            "roofline": {"kernel": ("ddx_schwarz_local_apply_sym" if pc.store.layout == "sym" else
                                    "ddx_schwarz_local_apply") + f" ({head}, R=1)", "bound": "hbm", "achieved": ach,
                         "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": ach / peaks["hbm_gbs"], "traffic": None,
                         "algorithmic_bytes": alg_bytes, "ms_per_launch": k_ms, "peak_source": peaks["source"]},
            "gpu_launches": launches, "clocks": clk,
            "setup_s": {"host": prob["host_setup_s"], "gpu": gpu_setup_s},
        }
    return out, prob, {"f64": {"iterations": spec["fp64_iterations"]}}


def run_ours(args, spec, rank: int, world: int):
    import torch
    import torch.distributed as dist

    import dd_solvers_b200 as dd
    from dd_solvers_b200 import _lib as L
    from dd_solvers_b200 import replicas

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    R = spec["R"]
    prob = build_problem(spec, device=dev)
    A = prob["A"]
    n = A.shape[0]
    At = dd.csr_to_torch(A).to(dev)
    head = args.precision
    precs = ("f64", "bf16", "f32", "f16") if R == 1 else ("f64", head)

    t0 = time.time()
    cls = dd.HybridSchwarz if spec["method"] == "hybrid" else dd.AdditiveSchwarz
    pc64 = cls(torch.float64, dd.Inv(), dd.CUDSS())
    pc64.setup(At, subdomains=(prob["sub_ptr"], prob["sub_idx"]), coarse_restriction=prob["R0"])
    pcs = {"f64": pc64}
    for name in precs[1:]:
        pcs[name] = pc64.requantize({"bf16": torch.bfloat16, "f32": torch.float32, "f16": torch.float16}[name])
    torch.cuda.synchronize()
    gpu_setup_s = time.time() - t0

    # one CG front-end per precision sharing the SELL matrix of the first
    base = dd.CG(None, rtol=1e-12, maxiter=2000, check_every=args.check_every)
    base.setup(At, block_size=1)
    mat = base.matrix

    def make(prec, rtol):
        cg = dd.CG(pcs[prec], rtol=rtol, maxiter=2000, check_every=args.check_every,
                   flexible=(prec != "f64"), replace_every=(args.replace_every if prec != "f64" else 0))
        cg.matrix = mat
        cg.n = n
        cg.block_size = 1
        return cg

    def rhs(step, nr=None):
        return torch.as_tensor(rhs_for(n, rank, step, spec, nr), device=dev)

    # FP64 reference solutions (single RHS at rtol 1e-12) for the checked columns
    check_cols = [0] if R == 1 else [0, R - 1]
    B0 = rhs(0, R)
    ref = {}
    for j in check_cols:
        bj = B0 if R == 1 else B0[:, j].contiguous()
        ref[j], _ = make("f64", 1e-12).solve(bj)

    def max_err(X):
        es = []
        for j in check_cols:
            xj = X if R == 1 else X[:, j]
            es.append(float(torch.linalg.norm(xj - ref[j]) / torch.linalg.norm(ref[j])))
        return max(es)

    # calibrate the stopping tolerance of each precision to reach 1e-8 error
    cal = {}
    for prec in precs:
        rtol = 1e-8
        for _ in range(6):
            cg = make(prec, rtol)
            if prec == "f64" and R > 1:
                x, meta = cg.solve(B0[:, 0].contiguous())  # FP64 plain comparison runs one RHS
                e = float(torch.linalg.norm(x - ref[0]) / torch.linalg.norm(ref[0]))
            else:
                x, meta = cg.solve(B0)
                e = max_err(x)
            if e <= 1e-8:
                break
            rtol /= 4
        its = meta["iterations"] if isinstance(meta["iterations"], int) else max(meta["iterations"])
        cal[prec] = {"rtol": rtol, "rel_error": e, "iterations": its, "solver": cg}

    steps, warm = args.steps, args.warmup

    def timed(prec, k, w, host=False, count_from_timed=False):
        cg = cal[prec]["solver"]
        nr = R if (prec != "f64" or R == 1) else 1
        bs = [rhs(s + 1, nr) for s in range(min(k, 4))]
        if host:
            bh = [b.cpu().pin_memory() for b in bs]
            xh = torch.empty_like(bh[0]).pin_memory()
            bd = torch.empty_like(bs[0])
        for s in range(w):
            cg.solve(bs[s % len(bs)])
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        its = []
        if count_from_timed:
            L.CALLS[0] = 0  # count only the kernels launched inside the timed region
        ev0.record()
        for s in range(k):
            if host:
                bd.copy_(bh[s % len(bh)], non_blocking=True)
                x, meta = cg.solve(bd)
                xh.copy_(x, non_blocking=True)
            else:
                x, meta = cg.solve(bs[s % len(bs)])
            its.append(meta["iterations"] if isinstance(meta["iterations"], int) else max(meta["iterations"]))
        ev1.record()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms = replicas.max_over_ranks(ev0.elapsed_time(ev1) / k, dev)
        return ms / nr, its  # per right-hand side

    clocks = Clocks(dev.index if dev.index is not None else 0)
    clocks.start()  # sampler running before the warm-up, so its start-up stays outside the timed region
    L.CALLS[0] = 0
    ms_head, its_head = timed(head, steps, warm, count_from_timed=True)
    clk = clocks.stop()
    launches = L.CALLS[0]
    # every timed solution meets the error bar
    errs = {}
    for prec in precs:
        nr = R if (prec != "f64" or R == 1) else 1
        bt = rhs(1, nr)
        x, _ = cal[prec]["solver"].solve(bt)
        es = []
        for j in (check_cols if nr > 1 else [0]):
            bj = bt if nr == 1 else bt[:, j].contiguous()
            xr, _ = make("f64", 1e-12).solve(bj)
            xj = x if nr == 1 else x[:, j]
            es.append(float(torch.linalg.norm(xj - xr) / torch.linalg.norm(xr)))
        errs[prec] = max(es)
    per_prec = {}
    for prec in precs:
        if prec == head:
            continue
        ms, its = timed(prec, max(1, min(steps, 3)), 1)
        per_prec[prec] = {"ms_per_rhs": ms, "iterations": its[-1], "rtol": cal[prec]["rtol"],
                          "rel_error": errs[prec]}
    per_prec[head] = {"ms_per_rhs": ms_head, "iterations": its_head[-1], "rtol": cal[head]["rtol"],
                      "rel_error": errs[head]}
    ms_e2e, _ = timed(head, steps, 1, host=True)

    # dominant kernel: local inverse apply of the head precision, timed alone
    # (200 launches, clocks sampled meanwhile, so the time can be read against
    # the SM clock the kernel ran at)
    pc = pcs[head]
    r = torch.randn(n * R, dtype=torch.float64, device=dev)
    for _ in range(3):
        pc._local(r, R)
    kev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    reps = 200
    kclk = Clocks(dev.index if dev.index is not None else 0, interval_ms=20)
    kclk.start()
    torch.cuda.synchronize()
    kev[0].record()
    for _ in range(reps):
        pc._local(r, R)
    kev[1].record()
    torch.cuda.synchronize()
    k_clk = kclk.stop()
    k_ms = kev[0].elapsed_time(kev[1]) / reps
    ks = pc.ks.astype(np.int64)
    elt = {"f64": 8, "f32": 4, "bf16": 2, "f16": 2}[head]
    tc = pc._tc_ok(R) and pc.use_tensor_cores
    # block bytes the kernel must stream: the full blocks (tensor-core path on
    # full blocks) or the stored upper-triangle tiles (SIMT path, symmetric
    # tensor-core path)
    tcsym = tc and pc._tc_config(R, pc._tc_terms(R))[0]
    if tc:
        blk_bytes = pc._tile_store(True).nbytes if tcsym else int((ks * ks).sum() * elt)
    else:
        blk_bytes = pc.store.nbytes
    alg_bytes = int(blk_bytes + 4 * len(ks) + ks.sum() * 4 + n * R * 8 + ks.sum() * R * 4)
    flops = float(2 * (ks * ks).sum() * R)
    # SpMV (FP64) timed alone too
    q = torch.empty_like(r)
    for _ in range(3):
        mat.launch(r, q, R, L.SPMV_PLAIN)
    torch.cuda.synchronize()
    kev[0].record()
    for _ in range(reps):
        mat.launch(r, q, R, L.SPMV_PLAIN)
    kev[1].record()
    torch.cuda.synchronize()
    s_ms = kev[0].elapsed_time(kev[1]) / reps
    spmv_bytes = mat.nnz * 12 + (n + 1) * 4 + n * R * 16

    # batched right-hand sides through the tensor-core local apply (single-RHS workloads)
    batched = None
    if args.batched and R == 1:
        Rb = args.batched
        cgb = make(head, cal[head]["rtol"])
        Bd = torch.as_tensor(np.stack([rhs_for(n, rank, 100 + j, spec) for j in range(Rb)], axis=1), device=dev)
        Xb, mb = cgb.solve(Bd)  # warm-up (builds tile store, captures graphs)
        ebs = []
        for j in (0, Rb - 1):
            xr, _ = make("f64", 1e-12).solve(Bd[:, j].contiguous())
            ebs.append(float(torch.linalg.norm(Xb[:, j] - xr) / torch.linalg.norm(xr)))
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        kb = max(1, min(steps, 3))
        e0.record()
        for _ in range(kb):
            Xb, mb = cgb.solve(Bd)
        e1.record()
        torch.cuda.synchronize()
        bms = replicas.max_over_ranks(e0.elapsed_time(e1) / kb, dev)
        rb = torch.randn(n * Rb, dtype=torch.float64, device=dev)
        pcb = pcs[head]
        # the solve's own form of the apply: without a pack pass when the x/r
        # update writes the B panels
        fused = cgb.fuse_panels and pcb.fused_pack_ok(Rb)
        if fused:
            pcb.pack_panels(rb, Rb)
        for _ in range(2):
            pcb._local(rb, Rb, packed=fused)
        torch.cuda.synchronize()
        kev[0].record()
        for _ in range(reps):
            pcb._local(rb, Rb, packed=fused)
        kev[1].record()
        torch.cuda.synchronize()
        tc_ms = kev[0].elapsed_time(kev[1]) / reps
        bsym, bstages = pcb._tc_config(Rb, pcb._tc_terms(Rb))
        tiles = pcb._tile_store(bsym)
        tc_blk = tiles.nbytes if bsym else int((ks * ks).sum() * elt)
        tc_bytes = tc_apply_bytes(pcb, Rb, tc_blk, n, fused)
        tc_flops = float(2 * (ks * ks).sum() * Rb)
        batched = {"rhs": Rb, "ms_per_solve": bms, "ms_per_rhs": bms / Rb, "iterations": max(mb["iterations"]),
                   "rel_error_vs_fp64_checked_columns": ebs,
                   "speedup_vs_fp64_plain_per_rhs": None,
                   "tc_kernel": {"name": "ddx_schwarz_local_apply_tc_sym" if bsym else "ddx_schwarz_local_apply_tc",
                                 "ms_per_launch": tc_ms,
                                 "algorithmic_bytes": tc_bytes, "tile_bytes": tiles.nbytes,
                                 "achieved_gbs": tc_bytes / (tc_ms * 1e-3) / 1e9,
                                 "hbm_frac": tc_bytes / (tc_ms * 1e-3) / 1e9 / load_peaks()["hbm_gbs"],
                                 "achieved_tflops": tc_flops / (tc_ms * 1e-3) / 1e12,
                                 "ring_stages": bstages,
                                 "mma_tflops": tc_mma_flops(pcb, Rb, bsym) / (tc_ms * 1e-3) / 1e12,
                                 "tensor_frac_of_measured_bf16_peak": tc_mma_flops(pcb, Rb, bsym) / (tc_ms * 1e-3)
                                 / 1e12 / load_peaks()["bf16_tflops"],
                                 "includes": ("tensor-core apply (the B panels are written by the x/r update)" if fused
                                              else "16-bit B-panel pack + tensor-core apply")}}

    peaks = load_peaks()
    out = None
    if rank == 0:
        ach = alg_bytes / (k_ms * 1e-3) / 1e9
        traffic = None
        tp = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tp):
            t = json.load(open(tp)).get(f"{args.workload}_local_apply_{head}_r{R}")
            if t:
                traffic = t["bytes_per_launch"]
        f64_ms = per_prec["f64"]["ms_per_rhs"]
        if batched is not None:
            batched["speedup_vs_fp64_plain_per_rhs"] = f64_ms / batched["ms_per_rhs"]
        kname = ("ddx_schwarz_local_apply_tc_sym" if tcsym else "ddx_schwarz_local_apply_tc") if tc else \
            ("ddx_schwarz_local_apply_sym" if pc.store.layout == "sym" else "ddx_schwarz_local_apply")
        out = {
            "metric": "time per RHS to 1e-8 rel. error (mixed-precision Schwarz PCG), 1 B200",
            "value": ms_head / world,
            "unit": "ms/RHS",
            "n_gpus": world,
            "steps": steps,
            "warmup": warm,
            "ms_per_step": ms_head * R,
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": f"{head} blocks / f32 accumulate / f64 PCG",
            "data": "synthetic (seeded coefficient fields and right-hand sides)",
            "config": {
                "workload": f"{args.workload}: {spec['name']}, {head} blocks",
                "n_dofs": n, "subdomains": prob["nparts"], "k_max": int(ks.max()), "k_min": int(ks.min()),
                "coarse_dofs": prob["R0"].shape[0], "rhs_per_step": R, "rtol_used": cal[head]["rtol"],
                "l2": "inputs larger than L2 (local inverse blocks %.1f GB per apply)" % (alg_bytes / 1e9),
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            },
            "rel_error_vs_fp64": errs[head],
            "iterations": its_head[-1],
            "blocks_shifted_to_stay_spd": len(pcs[head].store.shifted),
            "fp64_plain_ms_per_rhs": f64_ms,
            "speedup_vs_fp64_plain": f64_ms / ms_head,
            "per_precision": per_prec,
            "e2e": {"value": ms_e2e / world, "unit": "ms/RHS", "h2d_bytes_per_step": n * R * 8,
                    "d2h_bytes_per_step": n * R * 8},
            "roofline": {"kernel": f"{kname} ({head}, R={R})", "bound": "hbm", "achieved": ach,
                         "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": ach / peaks["hbm_gbs"],
                         "traffic": traffic, "algorithmic_bytes": alg_bytes, "ms_per_launch": k_ms,
                         "tflops": flops / (k_ms * 1e-3) / 1e12, "peak_source": peaks["source"],
                         "launches_timed": reps, "sm_mhz_while_timed": k_clk.get("sm_mhz"),
                         "clock_reasons_while_timed": k_clk.get("reasons"),
                         "ms_x_sm_mhz": (k_ms * k_clk["sm_mhz"]) if k_clk.get("sm_mhz") else None},
            "spmv_roofline": {"kernel": "ddx_spmv_sell_f64" if R == 1 else "ddx_spmv_csr_f64",
                              "achieved": spmv_bytes / (s_ms * 1e-3) / 1e9,
                              "frac": spmv_bytes / (s_ms * 1e-3) / 1e9 / peaks["hbm_gbs"], "ms_per_launch": s_ms,
                              "algorithmic_bytes": spmv_bytes},
            "gpu_launches": launches,
            "batched": batched,
            "clocks": clk,
            "setup_s": {"host": prob["host_setup_s"], "gpu": gpu_setup_s},
        }
    return out, prob, cal


# The reference's own logged run of its DG-SIPG experiment S10 / S8 / S8 (6.29M DOFs, hybrid Schwarz, FP64
# preconditioner with FP16 local blocks, CG rtol 1e-9) on an A100: results/experiment_precisions.csv, row
# "CG(HybridSchwarz(torch.float64, Inv(torch.float16), CUDSS), bsr_matmul=True)", min over 10 solves.
REFERENCE_EXPERIMENT = {"fine": "S10", "solvers": "S8", "coarse": "S8", "method": "hybrid", "precision": "f16",
                        "reference_iterations": 61, "reference_a100_ms_per_solve": 183.0207977294922}
# The same experiment at the higher degrees the reference logged (same file, same solver row): P3 on S9
# (5,242,880 DOFs, 10 per cell) and P5 on S8 (2,752,512 DOFs, 21 per cell), S8 subdomains and coarse cells.
REFERENCE_EXPERIMENTS_HIGHER_DEGREE = [
    {"degree": 3, "fine": "S9", "solvers": "S8", "coarse": "S8", "method": "hybrid", "precision": "f16",
     "reference_iterations": 131, "reference_a100_ms_per_solve": 457.8937683105469},
    {"degree": 5, "fine": "S8", "solvers": "S8", "coarse": "S8", "method": "hybrid", "precision": "f16",
     "reference_iterations": 151, "reference_a100_ms_per_solve": 451.76153564453125},
]


def reference_experiment() -> dict:
    """The same experiment through this package (its SIPG system restated by dd_solvers_b200.dg, solved
    through the drop-in API, timed like the reference: CUDA events, min over repeated solves, setup
    excluded)."""
    import torch

    from dd_solvers_b200 import dg_experiments

    torch.cuda.empty_cache()
    e = REFERENCE_EXPERIMENT
    r = dg_experiments.run(e["fine"], e["solvers"], e["coarse"], e["method"], e["precision"], reps=5)
    torch.cuda.empty_cache()
    higher = []
    for h in REFERENCE_EXPERIMENTS_HIGHER_DEGREE:
        try:
            q = dg_experiments.run(h["fine"], h["solvers"], h["coarse"], h["method"], h["precision"], reps=5,
                                   degree=h["degree"])
        except Exception as exc:  # reported in the line; the headline metric does not depend on it
            higher.append({"degree": h["degree"], "fine": h["fine"], "error": repr(exc)[:200]})
            continue
        finally:
            torch.cuda.empty_cache()
        higher.append({"degree": h["degree"], "fine": h["fine"], "dofs": q["dofs"], "iterations": q["iterations"],
                       "reference_iterations": h["reference_iterations"], "ms_per_solve": q["solve_ms_min"],
                       "reference_a100_ms_per_solve": h["reference_a100_ms_per_solve"],
                       "speedup_vs_reference_a100": h["reference_a100_ms_per_solve"] / q["solve_ms_min"]})
    return {"experiment": "reference DG-SIPG P1, fine S10 (6,291,456 DOFs), 131,072 subdomains of 48 DOFs, "
                          "131,072 P0 coarse DOFs, HybridSchwarz(float64, Inv(float16), CUDSS), CG rtol 1e-9",
            "iterations": r["iterations"], "reference_iterations": e["reference_iterations"],
            "ms_per_solve": r["solve_ms_min"], "reference_a100_ms_per_solve": e["reference_a100_ms_per_solve"],
            "speedup_vs_reference_a100": e["reference_a100_ms_per_solve"] / r["solve_ms_min"],
            "higher_degree": higher,
            "source": "results/experiment_precisions.csv (the reference's log)"}


def tc_mma_flops(pc, R: int, sym: bool) -> float:
    """Flops the tensor cores issue in one local apply: two products per
    off-diagonal upper-triangle 128 x 128 tile and one per diagonal tile
    (symmetric storage), or the 128-row x 64-column padded full blocks."""
    ks = pc.ks.astype(np.int64)
    if sym:
        nt = (ks + 127) // 128
        return float(2 * R * 128 * 128 * (nt * nt).sum())
    rows = (ks + 7) // 8 * 8
    cols = (ks + 63) // 64 * 64
    return float(2 * R * (rows * cols).sum())


def tc_apply_bytes(pc, R: int, blk_bytes: int, n: int, fused: bool) -> int:
    """Algorithmic bytes of one tensor-core local apply: the block tiles, the
    per-subdomain scales and sizes, the r input (the B panels it reads when the
    x/r update wrote them, else r itself, n R FP64 values) and the FP32 local
    products written."""
    ks = pc.ks.astype(np.int64)
    if fused:
        panels = int((2 * ((ks + 127) // 128) * 64 * 2 * R).sum())
        return int(blk_bytes + 4 * len(ks) + ks.sum() * 4 + panels + ks.sum() * R * 4)
    return int(blk_bytes + 4 * len(ks) + ks.sum() * 4 + n * R * 8 + ks.sum() * R * 4)


def time_ms(fn, reps: int = 10) -> float:
    import torch

    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def multi_rhs_summary(args, name: str, prec: str) -> dict:
    """Compact result of a multi-RHS workload (c3: 64 RHS, c5: 16 RHS) for the
    c2 line: ms per RHS of the block solve to <= 1e-8 error on the checked
    columns, iterations, the FP64 single-RHS path on the same problem, and the
    dominant kernels (tensor-core local apply with its HBM and tensor
    utilisation, multi-RHS SpMM) timed alone with CUDA events."""
    import torch

    import dd_solvers_b200 as dd
    from dd_solvers_b200 import _lib as L

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    spec = WORKLOADS[name]
    t0 = time.time()
    prob = build_problem(spec, device=dev)
    A = prob["A"]
    n, R = A.shape[0], spec["R"]
    At = dd.csr_to_torch(A).to(dev)
    cls = dd.HybridSchwarz if spec["method"] == "hybrid" else dd.AdditiveSchwarz
    pc64 = cls(torch.float64, dd.Inv(), dd.CUDSS())
    pc64.setup(At, subdomains=(prob["sub_ptr"], prob["sub_idx"]), coarse_restriction=prob["R0"])
    dt = {"bf16": torch.bfloat16, "f16": torch.float16}[prec]
    pcq = pc64.requantize(dt)
    setup_s = time.time() - t0
    base = dd.CG(None, rtol=1e-12, maxiter=3000)
    base.setup(At, block_size=1)

    def make(pc, rtol, flexible):
        cg = dd.CG(pc, rtol=rtol, maxiter=3000, check_every=args.check_every, flexible=flexible)
        cg.matrix, cg.n, cg.block_size = base.matrix, n, 1
        return cg

    B = torch.as_tensor(rhs_for(n, 0, 1, spec, R), device=dev)
    cols = [0, R - 1]
    ref = {j: make(pc64, 1e-12, False).solve(B[:, j].contiguous())[0] for j in cols}

    def err(X):
        return max(float(torch.linalg.norm(X[:, j] - ref[j]) / torch.linalg.norm(ref[j])) for j in cols)

    rtol = 1e-8
    for _ in range(5):
        cg = make(pcq, rtol, True)
        X, meta = cg.solve(B)
        e = err(X)
        if e <= 1e-8:
            break
        rtol /= 4
    k = max(1, min(args.steps, 3))
    ms = time_ms(lambda: cg.solve(B), k)
    its = max(meta["iterations"])
    # FP64 plain path, one RHS per solve, tolerance reaching 1e-8 error
    r64 = 1e-8
    for _ in range(5):
        cg64 = make(pc64, r64, False)
        x64, m64 = cg64.solve(B[:, 0].contiguous())
        if float(torch.linalg.norm(x64 - ref[0]) / torch.linalg.norm(ref[0])) <= 1e-8:
            break
        r64 /= 4
    ms64 = time_ms(lambda: cg64.solve(B[:, 0].contiguous()), 2)
    # dominant kernels alone
    peaks = load_peaks()
    r = torch.randn(n * R, dtype=torch.float64, device=dev)
    terms = pcq._tc_terms(R)
    sym, stages = pcq._tc_config(R, terms)
    fused = cg.fuse_panels and pcq.fused_pack_ok(R)
    if fused:
        pcq.pack_panels(r, R)
    k_ms = time_ms(lambda: pcq._local(r, R, packed=fused), 10)
    ks = pcq.ks.astype(np.int64)
    blk = pcq._tile_store(True).nbytes if sym else int((ks * ks).sum() * 2)
    alg = tc_apply_bytes(pcq, R, blk, n, fused)
    flops = tc_mma_flops(pcq, R, sym)
    q = torch.empty_like(r)
    mat = base.matrix
    s_ms = time_ms(lambda: mat.launch(r, q, R, L.SPMV_PLAIN), 10)
    s_bytes = mat.nnz * 12 + (n + 1) * 4 + n * R * 16
    out = {"workload": f"{name}: {spec['name']}, {prec} blocks", "rhs": R, "ms_per_rhs": ms / R,
           "ms_per_solve": ms, "iterations": its, "rtol_used": rtol, "rel_error_vs_fp64_checked_columns": e,
           "fp64_plain_ms_per_rhs": ms64, "fp64_plain_iterations": m64["iterations"],
           "speedup_vs_fp64_plain": ms64 / (ms / R), "setup_s": setup_s,
           "tc_kernel": {"name": "ddx_schwarz_local_apply_tc_sym" if sym else "ddx_schwarz_local_apply_tc",
                         "ring_stages": stages, "ms_per_launch": k_ms, "algorithmic_bytes": alg,
                         "achieved_gbs": alg / (k_ms * 1e-3) / 1e9, "hbm_frac": alg / (k_ms * 1e-3) / 1e9 /
                         peaks["hbm_gbs"], "mma_tflops": flops / (k_ms * 1e-3) / 1e12,
                         "tensor_frac_of_measured_bf16_peak": flops / (k_ms * 1e-3) / 1e12 / peaks["bf16_tflops"],
                         "includes": ("tensor-core apply (the B panels are written by the x/r update)" if fused
                                      else "16-bit B-panel pack + tensor-core apply")},
           "spmm": {"name": "ddx_spmv_csr_f64",
                    "ms_per_launch": s_ms, "algorithmic_bytes": s_bytes,
                    "hbm_frac": s_bytes / (s_ms * 1e-3) / 1e9 / peaks["hbm_gbs"]}}
    del cg, cg64, pcq, pc64, base, mat, ref, B, r, q
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return out


# Timed full CPU solves of the reference arm: as many of the requested steps as
# fit this many seconds (at least one); the line says how many were timed.
REF_BUDGET_S = 150.0


def _blocks_bytes(prob) -> int:
    """Host bytes the CPU solve holds for its FP64 blocks: the per-block list and,
    while it is stacked by block size, the stacked copy."""
    ks = np.diff(prob["sub_ptr"]).astype(np.int64)
    return int((ks * ks).sum() * 8) * 2


def _host_ram() -> int:
    try:
        import psutil

        return int(psutil.virtual_memory().available)
    except Exception:
        return 0


def reference_arm(args, spec) -> dict:
    """The reference arm: the FP64 CPU restatement of the path (the reference's
    own solver needs CUDA for its kernels and cuDSS; its algorithm on CPU is what
    the oracle restatement reproduces) on the host cores, on this arm's workload,
    metric and unit. One step = one full solve of one right-hand side to the
    tolerance the FP64 path needs for 1e-8 error; the inverse blocks are computed
    on the host first and excluded from the time, as the reference excludes
    setup. The timed steps stop once REF_BUDGET_S seconds have been spent."""
    prob = build_problem(spec)
    unit = "ms/gradient" if spec["kind"] == "grad" else "ms/RHS"
    if _blocks_bytes(prob) > 0.7 * _host_ram():
        return {"impl": "reference", "unavailable": f"the FP64 inverse blocks ({_blocks_bytes(prob) / 1e9:.0f} GB) "
                                                    f"exceed this host's free memory"}
    t0 = time.time()
    blocks = host_inverses(prob)
    setup_s = time.time() - t0
    per_value = 2 if spec["kind"] == "grad" else 1  # a gradient is a forward and an adjoint solve
    rtol = spec.get("fp64_rtol", 1e-8)
    vals, first = [], None
    t_start = time.time()
    for _ in range(max(1, args.steps)):
        cb = cpu_solve_per_rhs(prob, spec, rtol, blocks)
        first = first or cb
        vals.append(cb["ms_per_rhs"] * per_value)
        if time.time() - t_start > REF_BUDGET_S:
            break
    v = min(vals)
    sample = (first["sample"].replace("min over 1 solve(s)", f"min over {len(vals)} timed solves") +
              (" (x2: forward and adjoint solve per gradient)" if per_value == 2 else ""))
    return {"metric": "time per RHS to 1e-8 rel. error (mixed-precision Schwarz PCG), 1 B200",
            "value": v, "unit": unit, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "steps_timed": len(vals), "higher_is_better": False, "impl": "reference", "dtype": "f64",
            "config": {"workload": f"{args.workload}: {spec['name']}, FP64 CPU restatement"},
            "cpu_baseline": {"value": v, "unit": unit, "cores": first["cores"], "kind": "port", "sample": sample,
                             "setup_s": setup_s, "iterations": first["iterations"]},
            "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def cpu_baseline(spec, prob, cal, unit) -> dict:
    """cpu_baseline of the GPU line: full FP64 solves of the oracle restatement on
    the host cores with the GPU operator's FP64 inverse blocks (copied to the
    host; setup excluded), one right-hand side, min over two solves."""
    pc = cal.get("f64", {}).get("solver")
    pc = getattr(pc, "preconditioner", None)
    if pc is None or _blocks_bytes(prob) > 0.7 * _host_ram():
        blocks = None if _blocks_bytes(prob) > 0.7 * _host_ram() else host_inverses(prob)
    else:
        blocks = gpu_blocks_to_host(pc)
    if blocks is None:
        return {"value": None, "unit": unit, "cores": os.cpu_count(), "kind": "port",
                "sample": "not run: the FP64 inverse blocks exceed this host's free memory"}
    per_value = 2 if spec["kind"] == "grad" else 1
    cb = cpu_solve_per_rhs(prob, spec, cal.get("f64", {}).get("rtol", 1e-8), blocks, repeats=2)
    del blocks
    return {"value": cb["ms_per_rhs"] * per_value, "unit": unit, "cores": cb["cores"], "kind": "port",
            "sample": cb["sample"] + (" (x2: forward and adjoint solve per gradient)" if per_value == 2 else ""),
            "iterations": cb["iterations"]}


def other_workload_summary(args, name: str) -> dict:
    """Compact result of another configuration (c1: additive Schwarz on the 2D
    Poisson problem; c4: the differentiable solve) in the c2 line at N = 1, so
    that one default run records every configuration: its own runner with
    short timing (3 steps after 2 warm-up steps) and no CPU baseline."""
    import torch

    sub = argparse.Namespace(**vars(args))
    sub.workload, sub.steps, sub.warmup, sub.batched = name, 3, 2, 0
    spec = WORKLOADS[name]
    runner = run_grad if spec["kind"] == "grad" else run_ours
    res, _, cal = runner(sub, spec, 0, 1)
    torch.cuda.empty_cache()
    keep = ("metric", "value", "unit", "ms_per_step", "dtype", "iterations", "rel_error_vs_fp64",
            "fp64_plain_ms_per_rhs", "speedup_vs_fp64_plain", "fp64_blocks_ms_per_gradient",
            "speedup_vs_fp64_blocks", "gradient_check", "clocks")
    out = {k: res[k] for k in keep if k in res}
    out["workload"] = res["config"]["workload"]
    out["e2e"] = res["e2e"]["value"]
    out["dominant_kernel"] = {k: res["roofline"][k] for k in ("kernel", "ms_per_launch", "frac")}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="bf16", choices=["bf16", "f32", "f16"])
    ap.add_argument("--check-every", type=int, default=8)
    ap.add_argument("--replace-every", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batched", type=int, default=64, help="also time R right-hand sides per solve (0: skip)")
    ap.add_argument("--no-reference-experiment", action="store_true",
                    help="skip the reference's own DG experiment (run after the c2 measurement at N = 1)")
    ap.add_argument("--no-multi-rhs", dest="multi_rhs", action="store_false",
                    help="skip the compact c3 / c5 sub-results of the c2 line")
    ap.add_argument("--no-other-workloads", dest="other_workloads", action="store_false",
                    help="skip the compact c1 / c4 sub-results of the c2 line")
    args = ap.parse_args()
    spec = WORKLOADS[args.workload]

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))

    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps(reference_arm(args, spec)))
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    runner = run_grad if spec["kind"] == "grad" else run_ours
    out, prob, cal = runner(args, spec, rank, world)
    if rank == 0 and world == 1 and args.workload == "c2" and not args.no_reference_experiment:
        out["reference_experiment"] = reference_experiment()
    if rank == 0:
        if not args.no_cpu_baseline and world == 1:
            # the CPU baseline is measured at N = 1 only (the other ranks would wait on it)
            out["cpu_baseline"] = cpu_baseline(spec, prob, cal, out["unit"])
        if world == 1 and args.workload == "c2" and args.multi_rhs:
            cal.clear()
            torch.cuda.empty_cache()
            out["multi_rhs"] = {name: multi_rhs_summary(args, name, prec) for name, prec in
                                (("c3", "bf16"), ("c5", "f16"))}
        if world == 1 and args.workload == "c2" and args.other_workloads:
            cal.clear()
            torch.cuda.empty_cache()
            out["other_workloads"] = {name: other_workload_summary(args, name) for name in ("c1", "c4")}
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
