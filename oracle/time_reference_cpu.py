"""ORACLE (test infrastructure only): time the reference's own CPU solve beside
the restatement's, to calibrate the CPU baseline.

The reference cannot be shipped to a GPU host, so the timed CPU baseline there
is the restatement (``oracle/restatement.py``, batched mode). This script, run
where a checkout of the reference is available (``DDX_REFERENCE_ROOT``), times
on the same host cores and the same problem (config 1-R: Poisson 2D 256^2 cells,
15 x 15 equal subdomains of 17^2 DOFs in the reference's contiguous layout, P0
coarse space, one uniform right-hand side, rtol 1e-8):

* the reference's ``CG`` with ``AdditiveSchwarz`` / ``HybridSchwarz`` (``Inv``
  FP64 blocks), run verbatim on CPU tensors through ``oracle/ref_harness.py``,
  min over 5 solves, as ``experiments.py:252-272`` times a solve;
* the restatement in the layout the reference uses (``ContiguousSchwarz``) and in
  the index-set layout the CPU baseline runs (``Schwarz(batched=True)``), same
  rule.

Every solve uses all host threads for torch; NumPy's BLAS is held to one thread
(its idle workers otherwise contend with torch's). Prints one JSON line.

    DDX_REFERENCE_ROOT=<checkout> python -m oracle.time_reference_cpu
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np


def _min_time(fn, repeats=5):
    ts, out = [], None
    for _ in range(repeats):
        t0 = time.perf_counter()
        out = fn()
        ts.append(time.perf_counter() - t0)
    return min(ts), out


def main():
    import scipy.sparse as sps
    import torch
    from threadpoolctl import threadpool_limits

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from dd_solvers_b200 import partition, problems
    from oracle import ref_harness
    from oracle import restatement as orc

    S = ref_harness.load()
    torch.set_num_threads(os.cpu_count())
    P = problems.poisson2d(256)
    A = P.matrix
    n = A.shape[0]
    b = problems.uniform_rhs(n, seed=0)
    owner, nparts = partition.box_owner(P.interior_shape, 15)
    perm = np.argsort(owner, kind="stable")
    inv = np.empty_like(perm)
    inv[perm] = np.arange(n)
    At = torch.sparse_csr_tensor(torch.as_tensor(A.indptr.astype(np.int64)),
                                 torch.as_tensor(A.indices.astype(np.int64)), torch.as_tensor(A.data), A.shape)
    Ap = S.permute_csr_tensor(At, torch.as_tensor(inv))
    As = sps.csr_matrix((Ap.values().numpy(), Ap.col_indices().numpy(), Ap.crow_indices().numpy()), shape=(n, n))
    bp = torch.as_tensor(b[perm])
    sub_ptr, sub_idx = partition.overlapping_subdomains(A, owner, nparts, 0)
    R0 = partition.p0_restriction(owner, nparts)
    out = {"problem": "config 1-R: poisson2d 256^2 cells, 225 subdomains of 289 DOFs, P0 coarse, rtol 1e-8",
           "torch_threads": torch.get_num_threads(), "cores": os.cpu_count()}
    with threadpool_limits(1, user_api="blas"):
        for name, cls in (("additive", S.AdditiveSchwarz), ("hybrid", S.HybridSchwarz)):
            cg = S.CG(cls(torch.float64, S.Inv(), S.CUDSS()), rtol=1e-8, bsr_matmul=False)
            cg.setup(Ap, dofs_per_solver=289, solvers_per_coarse=torch.ones(nparts, dtype=torch.int64))
            t, (_, m) = _min_time(lambda: cg.solve(bp.clone()))
            out[f"reference_{name}"] = {"iterations": m["iterations"], "s_per_solve": t}

            Mc = orc.ContiguousSchwarz(As, 289, np.ones(nparts, dtype=np.int64))
            Ah = orc.HostCSR(As)
            apply = Mc.additive if name == "additive" else Mc.hybrid
            kw = {} if name == "additive" else {"T0": Mc.T0}
            t, (_, m) = _min_time(lambda: orc.pcg(Ah, b[perm], apply, rtol=1e-8, **kw))
            out[f"restatement_contiguous_{name}"] = {"iterations": m["iterations"], "s_per_solve": t}

            Ms = orc.Schwarz(A, sub_ptr, sub_idx, R0, batched=True)
            Ah = orc.HostCSR(A)
            apply = Ms.additive if name == "additive" else Ms.hybrid
            kw = {} if name == "additive" else {"T0": Ms.T0}
            t, (_, m) = _min_time(lambda: orc.pcg(Ah, b, apply, rtol=1e-8, **kw))
            out[f"restatement_index_sets_{name}"] = {"iterations": m["iterations"], "s_per_solve": t}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
