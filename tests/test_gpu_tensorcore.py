"""tcgen05 multi-RHS local apply: layout and numerics against the oracle.

The oracle applies the GPU's own dequantised blocks in FP64 to r rounded to
the block type in one or two 16-bit terms (what the tensor cores multiply),
so the only expected difference is FP32 accumulation: relative error <= 1e-5.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

from helpers import p1_case, q1_case, torch_csr

pytestmark = pytest.mark.gpu

DT = {"bf16": torch.bfloat16, "f16": torch.float16}


@pytest.mark.parametrize("variant", ["full", "sym"])
@pytest.mark.parametrize("terms", [1, 2])
@pytest.mark.parametrize("prec", ["bf16", "f16"])
@pytest.mark.parametrize("R", [16, 32, 64])
@pytest.mark.parametrize("case", ["q1_small", "q1_34sq", "p1_rcb"])
def test_tc_local_apply_matches_oracle(cuda, prec, R, case, terms, variant):
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
    pc.rhs_terms = terms
    pc.tc_symmetric = variant == "sym"
    pc.autotune = False  # the variant under test, not the tuner's choice
    if not pc._tc_ok(R):
        pytest.skip("subdomains too large for the shared-memory B panels at this R")
    if variant == "sym" and not pc._tc_sym_ok(R, terms):
        pytest.skip("accumulators of the largest block exceed TMEM, or full-block storage")
    rng = np.random.default_rng(R)
    r = rng.standard_normal((A.shape[0], R))
    rt = torch.as_tensor(r, device=cuda).contiguous()
    y = pc._local_sum(rt.view(-1), R).cpu().numpy()
    rq = orc.rhs_terms(r, prec, terms)
    for i in range(pc.n_solvers):
        idx = sub_idx[sub_ptr[i]:sub_ptr[i + 1]]
        ref = pc.store.block(i).cpu().numpy() @ rq[idx]
        got = y[sub_ptr[i]:sub_ptr[i + 1]]
        err = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-300)
        assert err <= 1e-5, (i, len(idx), err)


def test_two_residual_terms_approach_the_fp64_residual(cuda):
    """Against Q_i applied to the unrounded r, two BF16 terms cut the error by far more than 10x."""
    import dd_solvers_b200 as dd

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = p1_case(60, 8)
    pc = dd.AdditiveSchwarz(torch.float64, dd.Inv(torch.bfloat16), dd.CUDSS())
    pc.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0)
    r = np.random.default_rng(5).standard_normal((A.shape[0], 16))
    rt = torch.as_tensor(r, device=cuda).contiguous()
    errs = {}
    for terms in (1, 2):
        pc.rhs_terms = terms
        y = pc._local_sum(rt.view(-1), 16).cpu().numpy()
        num = den = 0.0
        for i in range(pc.n_solvers):
            idx = sub_idx[sub_ptr[i]:sub_ptr[i + 1]]
            ref = pc.store.block(i).cpu().numpy() @ r[idx]
            num += np.linalg.norm(y[sub_ptr[i]:sub_ptr[i + 1]] - ref) ** 2
            den += np.linalg.norm(ref) ** 2
        errs[terms] = (num / den) ** 0.5
    assert errs[2] < 1e-4 and errs[2] * 30 < errs[1], errs


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


@pytest.mark.parametrize("prec", ["bf16", "f16"])
def test_high_contrast_p1_tensor_cores_converge(cuda, prec):
    """Lognormal (sigma 1) jittered P1 blocks of ~2.4k DOFs, cond(A_i) ~ 1e4: the
    default term count reaches 1e-8 within 35% of the FP64-block iteration
    count (the oracle gives 91 FP64, 93 BF16 with two terms, 94-100 with one)."""
    import dd_solvers_b200 as dd
    from dd_solvers_b200 import partition, problems

    P = problems.p1_jittered(192, 0.3, 1.0, 3)
    A = P.matrix
    owner = partition.rcb_owner(P.coords, 16)
    sub_ptr, sub_idx = partition.overlapping_subdomains(A, owner, 16, 1)
    R0 = partition.p0_restriction(owner, 16)
    B = np.random.default_rng(2).standard_normal((A.shape[0], 16))
    Xd = spla.splu(A.tocsc()).solve(B)
    its = {}
    for p in ("f64", prec):
        dt = torch.float64 if p == "f64" else DT[p]
        cg = dd.CG(dd.HybridSchwarz(torch.float64, dd.Inv(dt), dd.CUDSS()), rtol=1e-10, replace_every=16)
        cg.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0, block_size=1)
        if p != "f64":
            assert cg.preconditioner._tc_ok(16)
        X, meta = cg.solve(torch.as_tensor(B, device=cuda))
        err = np.linalg.norm(X.cpu().numpy() - Xd, axis=0) / np.linalg.norm(Xd, axis=0)
        assert err.max() <= 1e-8, (p, err.max(), max(meta["iterations"]))
        its[p] = max(meta["iterations"])
    assert its[prec] <= 1.35 * its["f64"] + 2, its


def test_tc_symmetric_equals_full_blocks(cuda):
    """Symmetric-tile and full-block tensor-core kernels on the same blocks: same
    product up to FP32 accumulation order, on uneven RCB subdomains (k not a
    multiple of 128), in a multi-RHS PCG solve too."""
    import dd_solvers_b200 as dd

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = p1_case(100, 8)
    pc = dd.HybridSchwarz(torch.float64, dd.Inv(torch.float16), dd.CUDSS())
    pc.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0)
    pc.autotune = False
    assert pc._tc_sym_ok(16, 1) and int(pc.ks.max()) % 128 != 0
    r = torch.randn(A.shape[0], 16, dtype=torch.float64, device=cuda)
    ys = pc._local(r.view(-1), 16).clone()
    pc.tc_symmetric = False
    yf = pc._local(r.view(-1), 16).clone()
    rel = float(torch.linalg.norm(ys - yf) / torch.linalg.norm(yf))
    assert rel <= 1e-5, rel
    from dd_solvers_b200 import _lib

    assert _lib.device_error() == 0


@pytest.mark.parametrize("prec,terms", [("bf16", 1), ("bf16", 2), ("f16", 1)])
@pytest.mark.parametrize("R", [16, 32, 64])
def test_tc_every_tuning_candidate(cuda, prec, terms, R):
    """Every (symmetric / full tiles, ring depth) the tensor-core autotuner may
    pick, on uneven RCB subdomains (k not a multiple of 128, several row tiles)
    and on a 3D Q1 case (blocks of up to 1000 DOFs: 8 row tiles, all 512 TMEM
    columns at R = 64): each against the oracle, and the symmetric kernel bitwise
    equal for every ring depth (the depth changes no summation order)."""
    import dd_solvers_b200 as dd
    from dd_solvers_b200 import _lib
    from oracle import restatement as orc

    for case in ("p1", "q1_3d"):
        if case == "p1":
            P, A, owner, nparts, sub_ptr, sub_idx, R0 = p1_case(100, 8)
        else:
            P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(3, 32, 4, kappa_seed=3)
        pc = dd.AdditiveSchwarz(torch.float64, dd.Inv(DT[prec]), None)
        pc.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx))
        pc.rhs_terms = terms
        if not pc._tc_ok(R):
            continue
        cands = pc._tc_candidates(R, terms)
        rng = np.random.default_rng(R + terms)
        r = rng.standard_normal((A.shape[0], R))
        rt = torch.as_tensor(r, device=cuda).contiguous().view(-1)
        rq = orc.rhs_terms(r, prec, terms)
        s = pc.scratch(R)
        sym_out = None
        for sym, st in cands:
            s["ylocal"].zero_()
            pc._tc_apply(rt, s["ylocal"], R, terms, sym, st)
            y = s["ylocal"][: int(sub_ptr[-1]) * R].view(-1, R).double().cpu().numpy()
            for i in range(pc.n_solvers):
                idx = sub_idx[sub_ptr[i]:sub_ptr[i + 1]]
                ref = pc.store.block(i).cpu().numpy() @ rq[idx]
                got = y[sub_ptr[i]:sub_ptr[i + 1]]
                err = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-300)
                assert err <= 1e-5, (case, sym, st, i, err)
            if sym:
                if sym_out is None:
                    sym_out = y.copy()
                else:
                    assert np.array_equal(y, sym_out), (case, st)
        assert _lib.device_error() == 0
        best = pc.tune_tc(R)
        assert best in cands


@pytest.mark.parametrize("R", [16, 32, 64])
@pytest.mark.parametrize("prec", ["bf16", "f16"])
def test_update_xr_writes_the_packed_panels(cuda, R, prec):
    """ddx_pcg_update_xr_pack16_ex: x and r as the plain update computes them,
    the B panels bitwise equal to packing the new r (BF16: scale 1; FP16: the
    per-RHS scale of the squared norm the update started from, which it leaves
    in slot RR_PACK), ||r||^2 per column to rounding; overlapping 3D subdomains
    (DOFs in up to 8 panels)."""
    import dd_solvers_b200 as dd
    from dd_solvers_b200 import _lib as L
    from dd_solvers_b200.solvers import _PcgWork

    dt = torch.bfloat16 if prec == "bf16" else torch.float16
    P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(3, 24, 3, kappa_seed=2)
    pc = dd.HybridSchwarz(torch.float64, dd.Inv(dt), dd.CUDSS())
    pc.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0)
    pc.rhs_terms = 1
    assert pc.fused_pack_ok(R)
    n = A.shape[0]
    g = torch.Generator(device=cuda).manual_seed(R)
    x, p, r, q = (torch.randn(n * R, dtype=torch.float64, device=cuda, generator=g) for _ in range(4))
    w = _PcgWork(n, R, 10, cuda)
    L.call("ddx_pcg_reset", R, L.ptr(w.st), L.ptr(w.ist), 10, 0, 1e-8, 0.0, L.stream_ptr())
    alpha = torch.rand(R, dtype=torch.float64, device=cuda, generator=g)
    w.st.view(L.ST_COUNT, R)[L.ST_ALPHA] = alpha
    # the squared norms the update starts from: spread over many binades
    rr_old = torch.logspace(-30, 30, R, dtype=torch.float64, device=cuda)
    w.st.view(L.ST_COUNT, R)[L.ST_RR] = rr_old
    x0, r0 = x.clone(), r.clone()
    b16, _ = pc._panels(R, 1)
    b16.zero_()
    pan_ptr, pan_row = pc.panel_rows(R)
    L.call("ddx_pcg_update_xr_pack16_ex", n, R, L.ptr(x), L.ptr(r), L.ptr(p), L.ptr(q), L.ptr(pan_ptr),
           L.ptr(pan_row), L.ptr(b16), L.DTYPE_CODE[dt], L.ptr(w.st), L.ptr(w.ist), L.ptr(w.hist), L.ptr(w.partials),
           L.ptr(w.tickets), L.stream_ptr())
    fused = b16.clone()
    a = alpha.repeat(n)
    assert torch.allclose(x, x0 + a * p, rtol=1e-15, atol=1e-15)
    assert torch.allclose(r, r0 - a * q, rtol=1e-15, atol=1e-15)
    st = w.st.view(L.ST_COUNT, R)
    assert torch.allclose(st[L.ST_RR], (r.view(n, R) ** 2).sum(0), rtol=1e-12, atol=0)
    b16.zero_()
    if prec == "f16":
        assert torch.equal(st[L.ST_RR_PACK], rr_old)
        ref_st = torch.zeros_like(w.st)
        ref_st.view(L.ST_COUNT, R)[L.ST_RR] = rr_old
        pc.pack_panels(r, R, ref_st)
    else:
        pc.pack_panels(r, R)
    assert torch.equal(fused, b16)
    assert L.device_error() == 0


@pytest.mark.parametrize("R", [16, 64])
@pytest.mark.parametrize("prec", ["bf16", "f16"])
def test_fused_panel_solve_matches_unfused(cuda, R, prec):
    """Multi-RHS BF16 / FP16 tensor-core PCG with the panels written by the x/r
    update against the same solve with a pack pass: the same iterates (only the
    norms' summation order differs; FP16 panels scaled by a power of two from
    the previous norm, which changes no product), so the same iteration counts
    and solutions to rounding; with residual replacement too."""
    import dd_solvers_b200 as dd

    dt = torch.bfloat16 if prec == "bf16" else torch.float16
    P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(3, 24, 3, kappa_seed=4, coarse="q1")
    B = torch.as_tensor(np.random.default_rng(R).standard_normal((A.shape[0], R)), device=cuda)
    out = {}
    for fuse in (True, False):
        cg = dd.CG(dd.HybridSchwarz(torch.float64, dd.Inv(dt), dd.CUDSS()), rtol=1e-9,
                   replace_every=8)
        cg.fuse_panels = fuse
        cg.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0, block_size=1)
        cg.preconditioner.rhs_terms = 1
        out[fuse] = cg.solve(B)
    (X1, m1), (X0, m0) = out[True], out[False]
    assert all(abs(a - b) <= 1 for a, b in zip(m1["iterations"], m0["iterations"])), (m1["iterations"],
                                                                                         m0["iterations"])
    assert torch.allclose(X1, X0, rtol=0, atol=1e-9 * float(X0.abs().max()))
