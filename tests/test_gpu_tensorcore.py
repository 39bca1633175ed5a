"""tcgen05 multi-RHS local apply: layout and numerics against the oracle.

The oracle applies the GPU's own dequantised blocks in FP64 to r rounded to
the block type (what the tensor cores multiply), so the only expected
difference is FP32 accumulation: relative error <= 1e-5.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

from helpers import p1_case, q1_case, torch_csr

pytestmark = pytest.mark.gpu

DT = {"bf16": torch.bfloat16, "f16": torch.float16}


@pytest.mark.parametrize("prec", ["bf16", "f16"])
@pytest.mark.parametrize("R", [16, 32, 64])
@pytest.mark.parametrize("case", ["q1_small", "q1_34sq", "p1_rcb"])
def test_tc_local_apply_matches_oracle(cuda, prec, R, case):
    import dd_solvers_b200 as dd
    from oracle import restatement as orc

    if case == "q1_small":
        P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(2, 24, 3)
    elif case == "q1_34sq":
        P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(2, 96, 3)  # k up to 34^2 = 1156
    else:
        P, A, owner, nparts, sub_ptr, sub_idx, R0 = p1_case(60, 8)
    pc = dd.AdditiveSchwarz(torch.float64, dd.Inv(DT[prec]), dd.CUDSS())
    pc.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0)
    if not pc._tc_ok(R):
        pytest.skip("subdomains too large for the shared-memory B panel at this R")
    rng = np.random.default_rng(R)
    r = rng.standard_normal((A.shape[0], R))
    rt = torch.as_tensor(r, device=cuda).contiguous()
    y = pc._local(rt.view(-1), R).view(-1, R)[: len(sub_idx)].cpu().numpy()
    rq = orc.round_to(r, prec)
    for i in range(pc.n_solvers):
        idx = sub_idx[sub_ptr[i]:sub_ptr[i + 1]]
        ref = pc.store.block(i).cpu().numpy() @ rq[idx]
        got = y[sub_ptr[i]:sub_ptr[i + 1]]
        err = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-300)
        assert err <= 1e-5, (i, len(idx), err)


def test_tc_and_simt_agree(cuda):
    """Same blocks, SIMT per column (r read in FP64) vs tensor cores (r in BF16)."""
    import dd_solvers_b200 as dd

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(2, 64, 4)
    pc = dd.HybridSchwarz(torch.float64, dd.Inv(torch.bfloat16), dd.CUDSS())
    pc.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0)
    r = torch.randn(A.shape[0], 16, dtype=torch.float64, device=cuda)
    Z_tc = pc.solve(r)[0]
    pc.use_tensor_cores = False
    Z_simt = pc.solve(r)[0]
    rel = float(torch.linalg.norm(Z_tc - Z_simt) / torch.linalg.norm(Z_simt))
    assert rel < 1e-2  # r rounded to BF16 (2^-9 relative) in the tensor-core product


@pytest.mark.parametrize("prec", ["bf16", "f16"])
@pytest.mark.parametrize("R", [16, 64])
def test_multi_rhs_pcg_tensor_cores_reach_fp64_accuracy(cuda, prec, R):
    import dd_solvers_b200 as dd

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(3, 16, 4, kappa_seed=4, coarse="q1")
    B = np.random.default_rng(9).standard_normal((A.shape[0], R))
    lu = spla.splu(A.tocsc())
    Xd = lu.solve(B)
    cg = dd.CG(dd.HybridSchwarz(torch.float64, dd.Inv(DT[prec]), dd.CUDSS()), rtol=1e-10, replace_every=16)
    cg.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0, block_size=1)
    assert cg.preconditioner._tc_ok(R)
    X, meta = cg.solve(torch.as_tensor(B, device=cuda))
    err = np.linalg.norm(X.cpu().numpy() - Xd, axis=0) / np.linalg.norm(Xd, axis=0)
    assert err.max() <= 1e-8, (err.max(), max(meta["iterations"]))
