"""Pins the FP64 oracle restatement to the reference's own results (CPU only).

The fixtures were written by tests/golden/make_golden.py, which ran the
reference's CG / AdditiveSchwarz / HybridSchwarz (src/dd_solvers/dd_solvers/solvers.py)
on CPU through oracle/ref_harness.py.
"""
import numpy as np
import pytest
import scipy.sparse as sps

from conftest import golden
from oracle import restatement as orc


def _fixture24():
    g = golden("fixture24.npz")
    Ap = sps.csr_matrix((g["p_val"], g["p_col"], g["p_crow"]), shape=(24, 24))
    s2c = g["solvers_to_coarse"]
    spc = np.bincount(s2c)
    owner = np.repeat(np.arange(len(s2c)), 6)
    R0 = sps.csr_matrix((np.ones(24), (s2c[owner], np.arange(24))), shape=(len(spc), 24))
    sub_ptr = np.arange(len(s2c) + 1) * 6
    return g, Ap, R0, sub_ptr, np.arange(24)


@pytest.mark.parametrize("rhs_name", ["load", "rhs_u"])
@pytest.mark.parametrize("case", ["asm_f64", "hsm_f64", "none"])
def test_restatement_matches_reference_fixture24(rhs_name, case):
    g, Ap, R0, sub_ptr, sub_idx = _fixture24()
    b = g[rhs_name][g["perm"]]
    M = orc.Schwarz(Ap, sub_ptr, sub_idx, R0)
    if case == "asm_f64":
        x, meta = orc.pcg(Ap, b, M.additive, rtol=1e-12)
    elif case == "hsm_f64":
        x, meta = orc.pcg(Ap, b, M.hybrid, rtol=1e-12, T0=M.T0)
    else:
        x, meta = orc.pcg(Ap, b, None, rtol=1e-12)
    key = f"{rhs_name}__{case}"
    assert meta["iterations"] == int(g[key + "__iters"])
    xr = g[key + "__x"]
    assert np.linalg.norm(x - xr) <= 1e-10 * np.linalg.norm(xr)
    ref_norms = g[key + "__norms"]
    # histories agree to rounding amplification; the solution above is the pin.
    # Unpreconditioned CG runs past n iterations here, where rounding dominates.
    if case != "none":
        assert np.allclose(meta["residual norms"], ref_norms, rtol=1e-3, atol=1e-9 * ref_norms[0])


def test_restatement_inv32_matches_reference():
    """Reference Inv(float32) with FP64 vectors: blocks rounded to FP32, FP64 accumulate."""
    g, Ap, R0, sub_ptr, sub_idx = _fixture24()
    b = g["rhs_u"][g["perm"]]
    blocks = [orc.round_to(np.linalg.inv(Ap[i * 6:(i + 1) * 6, i * 6:(i + 1) * 6].toarray()), "f32")
              for i in range(4)]
    M = orc.Schwarz(Ap, sub_ptr, sub_idx, R0, inverse_blocks=blocks)
    x, meta = orc.pcg(Ap, b, M.hybrid, rtol=1e-12, T0=M.T0)
    assert meta["iterations"] == int(g["rhs_u__hsm_f64_inv32__iters"])
    xr = g["rhs_u__hsm_f64_inv32__x"]
    assert np.linalg.norm(x - xr) <= 1e-10 * np.linalg.norm(xr)


@pytest.mark.parametrize("batched", [False, True], ids=["per-block", "batched"])
def test_restatement_matches_reference_config1r(batched):
    """Both execution modes of the restatement (the per-block loop and the
    batched one the CPU baseline times: torch.bmm per block size, torch CSR
    products) reproduce the reference's iterates and iteration counts."""
    from dd_solvers_b200 import partition, problems

    g = golden("c1r.npz")
    P = problems.poisson2d(256)
    A = P.matrix
    b = problems.uniform_rhs(A.shape[0], seed=0)
    assert np.allclose(b[:16], g["b_head"])
    owner, nparts = partition.box_owner(P.interior_shape, 15)
    perm = np.argsort(owner, kind="stable")
    assert np.array_equal(perm[:64], g["perm_head"])
    sub_ptr, sub_idx = partition.overlapping_subdomains(A, owner, nparts, 0)
    R0 = partition.p0_restriction(owner, nparts)
    M = orc.Schwarz(A, sub_ptr, sub_idx, R0, batched=batched)
    Ah = orc.HostCSR(A) if batched else A
    for kind in ("asm_f64", "hsm_f64"):
        if kind == "asm_f64":
            x, meta = orc.pcg(Ah, b, M.additive, rtol=1e-8)
        else:
            x, meta = orc.pcg(Ah, b, M.hybrid, rtol=1e-8, T0=M.T0)
        assert meta["iterations"] == int(g[kind + "__iters"]), kind
        xr = g[kind + "__x"]
        assert np.linalg.norm(x[perm] - xr) <= 1e-10 * np.linalg.norm(xr), kind


def test_condition_estimate_matches_reference():
    g = golden("unit_cases.npz")
    A = sps.diags([0.5, 4.0, 21.0]).tocsr()
    # The reference test runs in float32 (torch.tensor default), which needs 6
    # iterations; in FP64 CG ends after 3. The estimate (42 = 21/0.5) agrees.
    x, meta = orc.pcg(A, np.ones(3), None, rtol=1e-9)
    assert meta["iterations"] == 3 and int(g["cond_iters"]) == 6
    # the reference pairs beta_i with alpha_{i-1}; betas[i-1] is the beta of iteration i
    assert np.isclose(orc.lanczos_condition(meta["alphas"], meta["betas"]), float(g["cond_estimate"]))


def test_convergence_quirk_raises_on_last_iteration():
    A = sps.diags([0.5, 4.0, 21.0]).tocsr()
    _, meta = orc.pcg(A, np.ones(3), None, rtol=1e-9)
    it = meta["iterations"]
    with pytest.raises(orc.ConvergenceNotAchieved):
        orc.pcg(A, np.ones(3), None, rtol=1e-9, maxiter=it + 1)
    orc.pcg(A, np.ones(3), None, rtol=1e-9, maxiter=it + 2)


def test_bf16_rounding_matches_torch():
    import torch

    x = np.random.default_rng(0).standard_normal(10000) * 10.0 ** np.random.default_rng(1).integers(-8, 8, 10000)
    t = torch.as_tensor(x).to(torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(orc.round_to_bf16(x), t)
    t16 = torch.as_tensor(x).to(torch.float32).to(torch.float16).to(torch.float64).numpy()
    assert np.array_equal(orc.round_to(x, "f16"), t16)


@pytest.mark.parametrize("dtype", ["f32", "bf16", "f16"])
def test_block_scale_rule(dtype):
    B = np.random.default_rng(2).standard_normal((20, 20)) * 3e-3
    s, Q = orc.quantize(B, dtype)
    assert np.log2(s) == int(np.log2(s))
    amax = np.abs(B / s).max()
    t = orc.TARGET_EXP[dtype]
    assert 2.0 ** (t - 1) < amax <= 2.0 ** t
