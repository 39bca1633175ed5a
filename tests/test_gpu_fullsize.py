"""Parity at the benchmark sizes.

* Config 1 exactly as stated (2D Q1 Poisson, 256^2 cells = 255^2 DOFs, U[-1,1]
  load from seed 0, 8 x 8 box subdomains with one layer of overlap, P0 coarse
  aggregates, additive Schwarz, FP64): the whole PCG solve against the oracle
  restatement, at equal iteration counts (1e-10 relative on the iterates x_1,
  x_10 and x_K, K the oracle's stopping iteration) and with the stopping
  iteration +-1.
* C2 / C3 / C5 at full size: every hot kernel once on the real operators,
  block sizes and index maps, against the oracle:
  - the system SpMV (SELL-32 for one RHS, CSR for R) against SciPy;
  - the FP64 local apply on sampled subdomains (the largest and the smallest
    block among them) against the symmetrised inverse of the oracle's local
    block ``A[idx][:, idx]``;
  - the low-precision block store against the oracle's quantisation of the same
    inverse (per-block scale, round to nearest: only entries whose two FP64
    inverses straddle a rounding boundary may differ, by one unit in the last
    place), and the low-precision apply (SIMT for one RHS, tcgen05 for R) against
    the stored blocks applied in FP64 to r rounded as the kernel rounds it;
  - the coarse solve against SciPy's sparse LU of R0 A R0^T.
"""
import numpy as np
import pytest
import scipy.sparse as sps
import scipy.sparse.linalg as spla
import torch

from helpers import torch_csr

pytestmark = pytest.mark.gpu

DT = {"bf16": torch.bfloat16, "f16": torch.float16, "f64": torch.float64}


def fixed_iterate(cg, b, K):
    """x_K: exactly K PCG iterations from x0 = 0 (rtol = atol = 0, maxiter = K)."""
    import dd_solvers_b200 as dd

    saved = (cg.rtol, cg.atol, cg.maxiter)
    cg.rtol, cg.atol, cg.maxiter = 0.0, 0.0, int(K)
    x0 = torch.zeros_like(b)
    try:
        with pytest.raises(dd.ConvergenceNotAchieved):
            cg.solve(b, x0=x0)
    finally:
        cg.rtol, cg.atol, cg.maxiter = saved
    return x0


def test_config1_as_stated_matches_oracle(cuda):
    import dd_solvers_b200 as dd
    from dd_solvers_b200.workloads import WORKLOADS, build_problem, rhs_for
    from oracle import restatement as orc

    spec = WORKLOADS["c1"]
    prob = build_problem(spec)
    A, sub_ptr, sub_idx, R0 = prob["A"], prob["sub_ptr"], prob["sub_idx"], prob["R0"]
    n = A.shape[0]
    assert n == 255 ** 2 and prob["nparts"] == 64 and R0.shape[0] == 64
    ks = np.diff(sub_ptr)
    assert ks.max() == 34 ** 2 and ks.min() == 32 ** 2  # 31-32 owned DOFs per axis + one overlap layer per side
    b = rhs_for(n, 0, 0, spec)
    assert b.min() >= -1 and b.max() <= 1
    M = orc.Schwarz(A, sub_ptr, sub_idx, R0)
    xo, om = orc.pcg(A, b, M.additive, rtol=1e-8, record_iterates=True)
    K = om["iterations"]
    cg = dd.CG(dd.AdditiveSchwarz(torch.float64, dd.Inv(), dd.CUDSS()), rtol=1e-8)
    cg.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0, block_size=1)
    bt = torch.as_tensor(b, device=cuda)
    x, meta = cg.solve(bt)
    assert abs(meta["iterations"] - K) <= 1, (meta["iterations"], K)
    k = min(len(meta["residual norms"]), len(om["residual norms"]))
    assert np.allclose(meta["residual norms"][:k], om["residual norms"][:k], rtol=1e-8)
    for kk in (1, 10, K):
        xk = fixed_iterate(cg, bt, kk).cpu().numpy()
        ref = om["iterates"][kk - 1]
        assert np.linalg.norm(xk - ref) <= 1e-10 * np.linalg.norm(ref), (kk, np.linalg.norm(xk - ref) /
                                                                        np.linalg.norm(ref))
    assert np.linalg.norm(x.cpu().numpy() - xo) <= 1e-10 * np.linalg.norm(xo)


# ---------------------------------------------------------------------------
# C2 / C3 / C5 at full size
# ---------------------------------------------------------------------------

@pytest.fixture(scope="module", params=["c2", "c3", "c5"])
def fullsize(request, cuda):
    """Problem + FP64 hybrid preconditioner of one workload (module scope: pytest
    groups the tests by workload, so each is built once and freed before the next)."""
    import dd_solvers_b200 as dd
    from dd_solvers_b200.workloads import WORKLOADS, build_problem

    torch.cuda.empty_cache()
    workload = request.param
    spec = WORKLOADS[workload]
    prob = build_problem(spec)
    At = torch_csr(prob["A"], cuda)
    pc = dd.HybridSchwarz(torch.float64, dd.Inv(), dd.CUDSS())
    pc.setup(At, subdomains=(prob["sub_ptr"], prob["sub_idx"]), coarse_restriction=prob["R0"])
    ks = np.diff(prob["sub_ptr"])
    n_s = 40 if ks.max() <= 1200 else 16
    pick = np.unique(np.concatenate([np.linspace(0, len(ks) - 1, n_s).astype(np.int64),
                                     [int(np.argmax(ks)), int(np.argmin(ks))]]))
    F = dict(name=workload, spec=spec, prob=prob, At=At, pc=pc, pick=pick, inv={})
    yield F
    F.clear()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def _oracle_inverse(F, i):
    """Symmetrised FP64 inverse of the oracle's local block of subdomain i."""
    from oracle import restatement as orc

    if i not in F["inv"]:
        p = F["prob"]
        idx = p["sub_idx"][p["sub_ptr"][i]:p["sub_ptr"][i + 1]]
        B = np.linalg.inv(orc.local_block(p["A"], idx))
        F["inv"][i] = 0.5 * (B + B.T)
    return F["inv"][i]


def test_fullsize_spmv(cuda, fullsize):
    from dd_solvers_b200.solvers import _SellMatrix

    F = fullsize
    workload = F["name"]
    A = F["prob"]["A"]
    M = _SellMatrix(F["At"])
    rng = np.random.default_rng(3)
    for R in sorted({1, F["spec"]["R"]}):
        x = rng.standard_normal((A.shape[0], R))
        y = (M @ torch.as_tensor(x if R > 1 else x[:, 0], device=cuda)).cpu().numpy().reshape(A.shape[0], R)
        ref = A @ x
        bound = abs(A) @ np.abs(x)  # rounding bound ~ nnz per row x eps x sum |a_ij x_j|
        assert np.all(np.abs(y - ref) <= 1e-13 * bound + 1e-300), (workload, R)


def test_fullsize_local_apply_fp64(cuda, fullsize):
    F = fullsize
    workload = F["name"]
    p, pc = F["prob"], F["pc"]
    r = np.random.default_rng(5).standard_normal(p["A"].shape[0])
    y = pc._local_sum(torch.as_tensor(r, device=cuda), 1).cpu().numpy()[:, 0]
    for i in F["pick"]:
        s0, s1 = p["sub_ptr"][i], p["sub_ptr"][i + 1]
        ref = _oracle_inverse(F, i) @ r[p["sub_idx"][s0:s1]]
        err = np.linalg.norm(y[s0:s1] - ref) / np.linalg.norm(ref)
        assert err <= 1e-10, (workload, int(i), int(s1 - s0), err)


def _ulp_diff(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """Distance in units of the last place between two 16-bit tensors of the same type."""
    ia = a.contiguous().view(torch.int16).to(torch.int32)
    ib = b.contiguous().view(torch.int16).to(torch.int32)
    # sign-magnitude -> ordered integers
    oa = torch.where(ia < 0, -(ia & 0x7FFF), ia)
    ob = torch.where(ib < 0, -(ib & 0x7FFF), ib)
    return (oa - ob).abs()


# (block precision, right-hand sides) checked per workload: the benchmark's own
LOWPREC = {"c2": [("bf16", 1), ("bf16", 64)], "c3": [("bf16", 64)], "c5": [("f16", 16), ("bf16", 16)]}


def test_fullsize_local_apply_lowprec(cuda, fullsize):
    F = fullsize
    qs = {}
    try:
        for prec, R in LOWPREC[F["name"]]:
            if prec not in qs:
                qs[prec] = F["pc"].requantize(DT[prec])
            _check_lowprec(cuda, F, qs[prec], prec, R)
    finally:
        qs.clear()
        torch.cuda.empty_cache()


def _check_lowprec(cuda, F, pcq, prec, R):
    from oracle import restatement as orc

    workload = F["name"]
    p = F["prob"]
    # (a) the store: per-block scale and rounding of the oracle's inverse; a
    # block re-rounded with a diagonal shift (its plain rounding was indefinite)
    # is checked to be positive definite instead
    for i in sorted(set(F["pick"].tolist()) | set(list(pcq.store.shifted)[:4])):
        if i in pcq.store.shifted:
            assert float(torch.linalg.eigvalsh(pcq.store.block(int(i))).min()) > 0, (workload, prec, int(i))
            continue
        Bo = _oracle_inverse(F, i)
        s_o = orc.block_scale(float(np.abs(Bo).max()), prec)
        s_g = float(pcq.store.scale[i])
        Qg = pcq.store.dense_q(int(i))
        Qo = torch.as_tensor(Bo / s_g, device=cuda).to(torch.float32).to(DT[prec])
        d = _ulp_diff(Qg, Qo)
        frac = float((d > 0).double().mean())
        assert s_g == s_o or abs(np.log2(s_g / s_o)) == 1, (int(i), s_g, s_o)
        assert int(d.max()) <= 1 and frac <= 1e-3, (workload, prec, int(i), int(d.max()), frac)
    # (b) the kernel: stored blocks applied in FP64 to r rounded as the kernel rounds it
    rng = np.random.default_rng(R)
    r = rng.standard_normal((p["A"].shape[0], R))
    rt = torch.as_tensor(r, device=cuda).contiguous()
    y = pcq._local_sum(rt.view(-1), R)
    terms = pcq._tc_terms(R) if pcq.use_tensor_cores else 0
    if R > 1:
        assert terms > 0, "the multi-RHS workloads run on the tensor cores"
    rq = orc.rhs_terms(r, prec, terms) if terms else r
    tol = 1e-5 if terms else 2e-6
    for i in F["pick"]:
        s0, s1 = p["sub_ptr"][i], p["sub_ptr"][i + 1]
        ref = pcq.store.block(int(i)).cpu().numpy() @ rq[p["sub_idx"][s0:s1]]
        got = y[s0:s1].cpu().numpy()
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err <= tol, (workload, prec, R, int(i), int(s1 - s0), err)


def test_fullsize_coarse_solve(cuda, fullsize):
    F = fullsize
    workload = F["name"]
    p, pc = F["prob"], F["pc"]
    A, R0 = p["A"], sps.csr_matrix(p["R0"])
    Ac = (R0 @ A @ R0.T).tocsc()
    nc = Ac.shape[0]
    for R in sorted({1, F["spec"]["R"]}):
        w = np.random.default_rng(R).standard_normal((nc, R))
        yc = torch.empty(nc * R, dtype=torch.float64, device=cuda)
        pc._coarse(torch.as_tensor(w, device=cuda).contiguous().view(-1), yc, R)
        ref = spla.splu(Ac).solve(w)
        got = yc.view(nc, R).cpu().numpy()
        assert np.linalg.norm(got - ref) <= 1e-10 * np.linalg.norm(ref), (workload, R)
