"""The benchmark workloads (the five configurations of the Schwarz-PCG path),
as seeded synthetic problems: matrix, subdomains and coarse restriction.

Used by ``bench.py`` and ``python -m dd_solvers_b200.microbench solve``.
"""
from __future__ import annotations

import time

import numpy as np

# fp64_iterations: PCG iterations of the FP64 method on the workload at the
# tolerance that reaches 1e-8 error (measured on B200 by the GPU arm; the CPU
# restatement reproduces it +-1; c4: forward + adjoint solve, from the
# restatement), the count the gradient workload reports for its FP64 solves.
# overlap: layers of overlap grown around each owned part (default 1).
WORKLOADS = {
    "c2": dict(kind="q1_3d", n_el=128, parts=16, coarse="q1", method="hybrid", rhs="uniform", R=1,
               fp64_iterations=31,
               name="hybrid-schwarz q1-3d 128^3 cells lognormal kappa, 4096 subdomains overlap 1, q1 coarse 3375"),
    "c1": dict(kind="q1_2d", n_el=256, parts=8, coarse="p0", method="additive", rhs="uniform", R=1,
               fp64_iterations=91,
               name="additive-schwarz q1-2d poisson 256^2 cells, 64 subdomains overlap 1, p0 coarse 64"),
    "c1r": dict(kind="q1_2d", n_el=256, parts=15, overlap=0, coarse="p0", method="hybrid", rhs="uniform", R=1,
                fp64_iterations=42,
                name="hybrid-schwarz q1-2d poisson 256^2 cells, 225 subdomains of 17^2 DOFs without overlap, "
                     "p0 coarse 225 (the reference's own layout: contiguous equal subdomains)"),
    "c3": dict(kind="q1_2d", n_el=1024, parts=32, coarse="p0", method="hybrid", rhs="normal", R=64,
               fp64_iterations=70,
               name="hybrid-schwarz q1-2d poisson 1024^2 cells, 1024 subdomains overlap 1, p0 coarse, 64 rhs"),
    "c4": dict(kind="grad", n_el=512, parts=16, coarse="p0", method="additive", rhs="ones", R=1,
               fp64_iterations=2 * 155,
               name="differentiable q1-2d 512^2 cells, kappa = exp(GRF l=0.1), f = 1, loss ||u - u_t||^2, "
                    "adjoint PCG + element gradient, additive schwarz 256 subdomains overlap 1, p0 coarse"),
    "c5": dict(kind="p1", n_nodes=2048, parts=2048, coarse="p0", method="hybrid", rhs="normal", R=16,
               fp64_iterations=139,
               name="hybrid-schwarz p1 jittered 2048^2 nodes lognormal kappa, rcb 2048 subdomains overlap 1, "
                    "p0 coarse, 16 rhs"),
}


def build_problem(spec: dict, seed: int = 0, device=None):
    """Matrix, owners, overlapping subdomains and coarse restriction of a
    workload (numpy / SciPy). With a CUDA ``device`` the RCB bisection and the
    overlap growth run there (``partition.rcb_owner_device``,
    ``overlapping_subdomains_device``: identical output, tested) and are copied
    back, and the coarse restriction ``R0`` is built there and stays there (a
    torch CSR; ``setup_ops.scipy_csr`` gives the SciPy copy)."""
    from . import partition, problems

    t0 = time.time()
    if spec["kind"] == "grad":
        g = problems.gaussian_random_field(spec["n_el"], 0.1, seed=seed)
        P = problems.q1_grid(2, spec["n_el"], np.exp(g))
        owner, nparts = partition.box_owner(P.interior_shape, spec["parts"])
    elif spec["kind"] == "q1_3d":
        P = problems.diffusion3d_lognormal(spec["n_el"], seed)
        owner, nparts = partition.box_owner(P.interior_shape, spec["parts"])
    elif spec["kind"] == "q1_2d":
        P = problems.poisson2d(spec["n_el"])
        owner, nparts = partition.box_owner(P.interior_shape, spec["parts"])
    else:
        P = problems.p1_jittered(spec["n_nodes"], 0.3, 1.0, seed)
        nparts = spec["parts"]
        if device is not None:
            import torch

            owner = partition.rcb_owner_device(torch.as_tensor(P.coords, device=device), nparts).cpu().numpy()
        else:
            owner = partition.rcb_owner(P.coords, nparts)
    A = P.matrix
    if device is not None:
        import torch

        crow = torch.as_tensor(A.indptr.astype(np.int64), device=device)
        col = torch.as_tensor(A.indices.astype(np.int64), device=device)
        sp, si = partition.overlapping_subdomains_device(crow, col, torch.as_tensor(owner, device=device), nparts,
                                                         spec.get("overlap", 1))
        sub_ptr, sub_idx = sp.cpu().numpy(), si.cpu().numpy()
    else:
        sub_ptr, sub_idx = partition.overlapping_subdomains(A, owner, nparts, spec.get("overlap", 1))
    if device is not None:
        import torch

        if spec["coarse"] == "q1":
            R0 = partition.q1_coarse_restriction_device(3, spec["n_el"], spec["parts"], device)
        else:
            R0 = partition.p0_restriction_device(torch.as_tensor(owner, device=device), nparts)
    elif spec["coarse"] == "q1":
        R0 = partition.q1_coarse_restriction(3, spec["n_el"], spec["parts"])
    else:
        R0 = partition.p0_restriction(owner, nparts)
    return dict(P=P, A=A, owner=owner, nparts=nparts, sub_ptr=sub_ptr, sub_idx=sub_idx, R0=R0,
                host_setup_s=time.time() - t0)


def rhs_for(n: int, rank: int, step: int, spec: dict, R: int | None = None):
    from . import problems, replicas

    seed = replicas.rhs_seed(rank, step)
    gen = problems.uniform_rhs if spec["rhs"] == "uniform" else problems.normal_rhs
    return gen(n, seed=seed, nrhs=R if (R or 1) > 1 else None)
