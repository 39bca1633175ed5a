"""Domain-sharded Schwarz PCG on one GPU: the ranks' shards run in one process
(LocalComm: exchanges are copies, sums add the shards in rank order; no kernel
waits on another shard), against the one-GPU solver and the oracle."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

from helpers import p1_case, q1_case, torch_csr

pytestmark = pytest.mark.gpu


def _case(name):
    if name == "q1_2d_p0":
        return q1_case(2, 48, 6)
    if name == "q1_3d_q1coarse":
        return q1_case(3, 16, 4, kappa_seed=5, coarse="q1")
    return p1_case(50, 16)


@pytest.mark.parametrize("case", ["q1_2d_p0", "q1_3d_q1coarse", "p1_rcb"])
@pytest.mark.parametrize("method", ["additive", "hybrid"])
@pytest.mark.parametrize("world", [2, 3])
def test_sharded_fp64_matches_one_gpu_and_oracle(cuda, case, method, world):
    import dd_solvers_b200 as dd
    from dd_solvers_b200.sharding import LocalComm, ShardedCG
    from oracle import restatement as orc

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = _case(case)
    b = np.random.default_rng(7).uniform(-1, 1, A.shape[0])
    bt = torch.as_tensor(b, device=cuda)
    sh = ShardedCG(method, torch.float64, rtol=1e-12, maxiter=2000)
    sh.setup(A, sub_ptr, sub_idx, owner, nparts, R0, comm=LocalComm(world), device=cuda)
    xs, ms = sh.solve(bt)
    cls = dd.AdditiveSchwarz if method == "additive" else dd.HybridSchwarz
    cg = dd.CG(cls(torch.float64, dd.Inv(), dd.CUDSS()), rtol=1e-12, maxiter=2000)
    cg.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0, block_size=1)
    x1, m1 = cg.solve(bt)
    assert abs(ms["iterations"] - m1["iterations"]) <= 1, (ms["iterations"], m1["iterations"])
    M = orc.Schwarz(A, sub_ptr, sub_idx, R0)
    if method == "additive":
        xr, om = orc.pcg(A, b, M.additive, rtol=1e-12, maxiter=2000)
    else:
        xr, om = orc.pcg(A, b, M.hybrid, rtol=1e-12, maxiter=2000, T0=M.T0)
    assert abs(ms["iterations"] - om["iterations"]) <= 1
    err = np.linalg.norm(xs.cpu().numpy() - xr) / np.linalg.norm(xr)
    assert err <= 1e-10, err
    # the residual history follows the one-GPU solve while rounding is far below it
    h_s, h_1 = np.array(ms["residual norms"]), np.array(m1["residual norms"])
    k = int(np.argmax(h_1 < 1e-6 * h_1[0])) if (h_1 < 1e-6 * h_1[0]).any() else len(h_1)
    assert np.allclose(h_s[:k], h_1[:k], rtol=1e-7, atol=0)


@pytest.mark.parametrize("prec", [torch.bfloat16, torch.float16, torch.float32])
def test_sharded_mixed_precision_multi_rhs_reaches_fp64_accuracy(cuda, prec):
    from dd_solvers_b200.sharding import LocalComm, ShardedCG

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = _case("q1_3d_q1coarse")
    B = np.random.default_rng(2).standard_normal((A.shape[0], 16))
    sh = ShardedCG("hybrid", prec, rtol=1e-10, maxiter=2000)
    sh.setup(A, sub_ptr, sub_idx, owner, nparts, R0, comm=LocalComm(2), device=cuda)
    X, meta = sh.solve(torch.as_tensor(B, device=cuda))
    Xd = spla.spsolve(A.tocsc(), B)
    err = np.linalg.norm(X.cpu().numpy() - Xd, axis=0) / np.linalg.norm(Xd, axis=0)
    assert err.max() <= 1e-8, (err.max(), meta["iterations"])


def test_sharded_one_rank_matches_unsharded(cuda):
    """world = 1: the shard is the whole problem, so the run takes the one-GPU
    solver's steps (the coarse products come from SciPy here and cuSPARSE
    there, so agreement is to rounding, not bits)."""
    import dd_solvers_b200 as dd
    from dd_solvers_b200.sharding import LocalComm, ShardedCG

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = _case("q1_2d_p0")
    bt = torch.as_tensor(np.random.default_rng(9).uniform(-1, 1, A.shape[0]), device=cuda)
    sh = ShardedCG("hybrid", torch.float64, rtol=1e-10)
    sh.setup(A, sub_ptr, sub_idx, owner, nparts, R0, comm=LocalComm(1), device=cuda)
    xs, ms = sh.solve(bt)
    cg = dd.CG(dd.HybridSchwarz(torch.float64, dd.Inv(), dd.CUDSS()), rtol=1e-10)
    cg.preconditioner.max_parts = 1
    cg.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0, block_size=1)
    cg.preconditioner.mapped_restriction = False
    x1, m1 = cg.solve(bt)
    assert ms["iterations"] == m1["iterations"]
    h_s, h_1 = np.array(ms["residual norms"]), np.array(m1["residual norms"])
    k = int(np.argmax(h_1 < 1e-6 * h_1[0])) if (h_1 < 1e-6 * h_1[0]).any() else len(h_1)
    assert np.allclose(h_s[:k], h_1[:k], rtol=1e-9, atol=0)
    assert torch.allclose(xs, x1, rtol=0, atol=1e-10 * float(x1.abs().max()))
