"""GPU parity of the individual kernels against the oracle / reference known answers.

Mirrors the reference's kernel tests: tests/test_gemv.py (7 dtype pairs x k,
rtol = atol = 1e-5), tests/test_bsr.py (fixture + random BSR, atol 1e-12 FP64 /
1e-6 FP32), tests/test_cusparse.py and tests/test_cudss.py (known answers).
"""
import numpy as np
import pytest
import scipy.sparse as sps
import torch

from conftest import golden
from helpers import p1_case, q1_case, torch_csr

pytestmark = pytest.mark.gpu

DT = {"f16": torch.float16, "bf16": torch.bfloat16, "f32": torch.float32, "f64": torch.float64}


@pytest.mark.parametrize("mat_dtype,vec_dtype", [("f16", "f32"), ("f16", "f64"), ("bf16", "f32"), ("bf16", "f64"),
                                                 ("f32", "f32"), ("f32", "f64"), ("f64", "f64")])
@pytest.mark.parametrize("k", [1, 2, 5, 10, 20, 50, 100, 200])
@pytest.mark.parametrize("use_shared_memory", [True, False])
def test_gemv_strided_batched(cuda, mat_dtype, vec_dtype, k, use_shared_memory):
    from dd_solvers_b200 import gemv_strided_batched

    n = 7
    rng = np.random.default_rng(42 + k)
    A = torch.as_tensor(rng.standard_normal((n, k, k))).to(DT[mat_dtype])
    A = A.permute(0, 2, 1).contiguous().permute(0, 2, 1).to(cuda)  # column-major
    b = torch.as_tensor(rng.standard_normal((n, k))).to(DT[vec_dtype]).to(cuda)
    exact = (A.to(b.dtype) @ b[:, :, None]).reshape(n, k)
    out = gemv_strided_batched(A, b, use_shared_memory=use_shared_memory)
    assert out.dtype == b.dtype
    assert torch.allclose(exact, out, rtol=1e-5, atol=1e-5)


def test_gemv_rejects_double_float(cuda):
    from dd_solvers_b200 import gemv_strided_batched

    A = torch.zeros(2, 3, 3, dtype=torch.float64, device=cuda).transpose(1, 2)
    with pytest.raises(RuntimeError, match="Double-Float"):
        gemv_strided_batched(A, torch.zeros(2, 3, dtype=torch.float32, device=cuda))


def _allclose(a, b):
    atol = 1e-6 if a.dtype == torch.float32 else 1e-12
    return torch.allclose(a, b, atol=atol)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_bsr_small_fixture(cuda, dtype):
    from dd_solvers_b200 import FastBSR

    g = golden("unit_cases.npz")
    m = torch.sparse_bsr_tensor(torch.as_tensor(g["bsr_crow"]), torch.as_tensor(g["bsr_col"]),
                                torch.as_tensor(g["bsr_val"]), size=g["bsr_dense"].shape).to(cuda, dtype)
    x = torch.randn(m.shape[0], device=cuda, dtype=dtype)
    y = FastBSR(m) @ x
    assert _allclose(y, torch.as_tensor(g["bsr_dense"], device=cuda, dtype=dtype) @ x)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("bs", [1, 2, 3, 4, 6, 8, 10, 11, 15, 16, 20, 21, 24])
def test_bsr_random(cuda, dtype, bs):
    from dd_solvers_b200 import FastBSR

    torch.manual_seed(bs)
    nbr, per = 1001, 3  # not a multiple of the block rows per warp
    crow = torch.arange(0, nbr * per + 1, per)
    col = torch.randint(0, nbr, (nbr * per,))
    vals = torch.randn(nbr * per, bs, bs, dtype=dtype)
    m = torch.sparse_bsr_tensor(crow, col, vals, size=(nbr * bs, nbr * bs))
    x = torch.randn(nbr * bs, dtype=dtype)
    # exact product of the same inputs; rounding bound ~ terms x eps x sum |a_ij x_j|
    dense = m.to_dense().double()
    expected = (dense @ x.double()).to(cuda)
    scale = (dense.abs() @ x.double().abs()).to(cuda)
    y = FastBSR(m.to(cuda)) @ x.to(cuda)
    eps = 1e-5 if dtype == torch.float32 else 1e-13
    assert torch.all((y.double() - expected).abs() <= eps * scale + 1e-300)


def test_csr_to_bsr_layout(cuda):
    from dd_solvers_b200 import csr_to_bsr

    m = torch.sparse_csr_tensor(torch.tensor([0, 2, 3, 5, 9]), torch.tensor([0, 1, 1, 0, 2, 0, 1, 2, 3]),
                                torch.tensor([1, 2, 3, 4, 5, 6, 7, 8, 9], dtype=torch.float64)).to(cuda)
    b = csr_to_bsr(m, 2)
    assert b.crow_indices().tolist() == [0, 1, 3]
    assert b.col_indices().tolist() == [0, 0, 1]
    assert b.values().stride() == (4, 1, 2)
    assert torch.equal(b.to_dense(), m.to_dense())


def test_cusparse_known_answers(cuda):
    from dd_solvers_b200 import gather_csr, sort_csr

    g = golden("unit_cases.npz")
    for i in range(int(g["n_cusparse_cases"])):
        tag = "sort" if f"sort{i}_in_crow" in g.files else "gather"
        fi = torch.sparse_csr_tensor(*(torch.as_tensor(g[f"{tag}{i}_in_{p}"]) for p in ("crow", "col", "val")),
                                     size=(len(g[f"{tag}{i}_in_crow"]) - 1, 4)).to(cuda)
        out = (sort_csr if tag == "sort" else gather_csr)(fi)
        for p, t in (("crow", out.crow_indices()), ("col", out.col_indices()), ("val", out.values())):
            assert np.array_equal(t.cpu().numpy(), g[f"{tag}{i}_out_{p}"]), (tag, i, p)


@pytest.mark.parametrize("value_type", [torch.float32, torch.float64])
def test_cudss_known_answers(cuda, value_type):
    from dd_solvers_b200 import cudss

    g = golden("unit_cases.npz")
    A = torch.sparse_csr_tensor(torch.as_tensor(g["spd_3x3_crow"]), torch.as_tensor(g["spd_3x3_col"]),
                                torch.as_tensor(g["spd_3x3_val"]).to(value_type), size=(3, 3)).to(cuda)
    s = cudss.spd_factorize(A)
    for xn, bn in (("cudss_x1", "cudss_b1"), ("cudss_x2", "cudss_b2")):
        x = s.solve(torch.as_tensor(g[bn], device=cuda, dtype=value_type))
        assert x.dtype == value_type
        assert torch.allclose(x, torch.as_tensor(g[xn], device=cuda, dtype=value_type), atol=1e-6)
    # batch: block-diagonal 3x3 + 2x2
    nrows = torch.tensor([3, 2])
    nnz = torch.tensor([5, 4])
    vals = torch.cat([torch.as_tensor(g["spd_3x3_val"]), torch.as_tensor(g["spd_2x2_val"])]).to(value_type)
    cols = torch.cat([torch.as_tensor(g["spd_3x3_col"]), torch.as_tensor(g["spd_2x2_col"])])
    rows = torch.cat([torch.as_tensor(g["spd_3x3_crow"]), torch.as_tensor(g["spd_2x2_crow"])])
    bs = cudss.spd_batch_factorize(nrows, nnz, vals.to(cuda), cols.to(cuda), rows.to(cuda))
    x = bs.solve(torch.as_tensor(g["cudss_b"], device=cuda, dtype=value_type))
    assert torch.allclose(x, torch.as_tensor(g["cudss_x"], device=cuda, dtype=value_type), atol=1e-6)


# ---------------------------------------------------------------------------
# SpMV (SELL-32 and CSR multi-RHS) vs SciPy
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("case", ["q1_2d", "q1_3d", "p1"])
@pytest.mark.parametrize("R", [1, 4, 64])
def test_spmv(cuda, case, R):
    from dd_solvers_b200.solvers import _SellMatrix

    if case == "q1_2d":
        A = q1_case(2, 40)[1]
    elif case == "q1_3d":
        A = q1_case(3, 12, kappa_seed=1)[1]
    else:
        A = p1_case(40)[1]
    M = _SellMatrix(torch_csr(A, cuda))
    rng = np.random.default_rng(R)
    x = rng.standard_normal((A.shape[0], R))
    y = (M @ torch.as_tensor(x if R > 1 else x[:, 0], device=cuda)).cpu().numpy().reshape(A.shape[0], R)
    ref = A @ x
    assert np.max(np.abs(y - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("case", ["q1_2d", "q1_3d", "p1"])
@pytest.mark.parametrize("R", [2, 16, 64])
@pytest.mark.parametrize("cluster", [8, 64, 200])
def test_spmm_cluster_order_same_rows(cuda, case, R, cluster):
    """The SpMM in breadth-first cluster order (ddx_spmv_csr_ordered_f64) gives
    every row of A x with the same bits as the row-order kernel (a row's sum
    does not depend on the work order); its fused p.q (PQ mode) agrees to
    rounding. The order is a permutation of the rows."""
    from dd_solvers_b200 import _lib as L
    from dd_solvers_b200.solvers import _PcgWork, _SellMatrix

    if case == "q1_2d":
        A = q1_case(2, 40)[1]
    elif case == "q1_3d":
        A = q1_case(3, 12, kappa_seed=1)[1]
    else:
        A = p1_case(40)[1]
    n = A.shape[0]
    M = _SellMatrix(torch_csr(A, cuda))
    M.spmm_cluster = cluster
    chunk = M._chunk_for(R)
    assert chunk % (512 // R) == 0 and chunk >= cluster
    order = M.row_order(chunk).cpu().numpy()
    assert np.array_equal(np.sort(order), np.arange(n))
    x = torch.randn(n * R, dtype=torch.float64, device=cuda)
    outs, pq = [], []
    for cl in (0, cluster):
        M.spmm_cluster = cl
        y = torch.full_like(x, float("nan"))
        M.launch(x, y, R, L.SPMV_PLAIN)
        outs.append(y)
        w = _PcgWork(n, R, 4, cuda)
        L.call("ddx_pcg_reset", R, L.ptr(w.st), L.ptr(w.ist), 4, 0, 1e-8, 0.0, L.stream_ptr())
        M.launch(x, w.q, R, L.SPMV_PQ, w)
        pq.append(w.st.view(L.ST_COUNT, R)[L.ST_PQ].clone())
    assert torch.equal(outs[0], outs[1])
    assert torch.allclose(pq[0], pq[1], rtol=1e-13, atol=0)


@pytest.mark.parametrize("prec", ["f64", "bf16"])
@pytest.mark.parametrize("R", [4, 16])
def test_mapped_restriction_bitwise_equal(cuda, prec, R):
    """Hybrid Schwarz with R >= 2: the restriction that reads y through the
    transpose map gives the same preconditioned vector, bit for bit, as the
    path that first writes y (overlapping Q1 subdomains: DOFs in 1-4 local
    products; SIMT and tensor-core local applies)."""
    import dd_solvers_b200 as dd

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(2, 48, 6)
    pc = dd.HybridSchwarz(torch.float64, dd.Inv(DT[prec]), dd.CUDSS())
    pc.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0)
    pc.sub_restriction = False
    r = torch.randn(A.shape[0], R, dtype=torch.float64, device=cuda)
    pc.mapped_restriction = True
    z1 = pc.solve(r)[0]
    pc.mapped_restriction = False
    z0 = pc.solve(r)[0]
    assert torch.equal(z0, z1)


@pytest.mark.parametrize("case", ["q1_2d_p0", "q1_3d_q1", "p1_rcb"])
@pytest.mark.parametrize("R", [2, 16, 64])
@pytest.mark.parametrize("slices", [1, 3])
def test_sub_restriction_kernel_matches_scipy(cuda, case, R, slices):
    """ddx_schwarz_restrict_sub on FP32 and FP64 local products: A_R y with
    y = sum_i R_i^T ylocal_i (summed over ylocal's slices), against SciPy in
    FP64 (P0 and Q1 coarse spaces, overlapping boxes and RCB parts); two calls
    in a row give the same bits."""
    from dd_solvers_b200 import _lib as L
    from dd_solvers_b200 import setup_ops as so

    if case == "q1_2d_p0":
        P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(2, 48, 6)
    elif case == "q1_3d_q1":
        P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(3, 12, 3, kappa_seed=2, coarse="q1")
    else:
        P, A, owner, nparts, sub_ptr, sub_idx, R0 = p1_case(40, 16)
    AR = sps.csr_matrix(R0 @ A)
    AR.sort_indices()
    n_c, n = AR.shape
    sp = torch.as_tensor(sub_ptr, device=cuda)
    plan = so.subdomain_restriction(torch.as_tensor(AR.indptr.astype(np.int64), device=cuda),
                                    torch.as_tensor(AR.indices.astype(np.int32), device=cuda),
                                    torch.as_tensor(AR.data, device=cuda), n_c, n, sp,
                                    torch.as_tensor(sub_idx, device=cuda), slices=slices)
    assert plan["max_slots"] <= so.RESTRICT_MAX_SLOTS
    total = int(sub_ptr[-1])
    for acc in (torch.float32, torch.float64):
        yl = torch.randn(slices * total, R, dtype=torch.float64, device=cuda).to(acc)
        part = torch.empty(plan["n_pairs"] * R, dtype=torch.float64, device=cuda)
        outs = []
        for _ in range(2):
            w = torch.full((n_c * R,), float("nan"), dtype=torch.float64, device=cuda)
            L.call("ddx_schwarz_restrict_sub", len(sub_ptr) - 1, plan["n_pairs"], n_c, R, L.ptr(sp),
                   L.ptr(plan["slot_base"]), L.ptr(plan["n_slots"]), L.ptr(plan["f_slot"]), L.ptr(plan["f_val"]),
                   L.ptr(plan["ov_ptr"]), L.ptr(plan["ov_slot"]), L.ptr(plan["ov_val"]), L.ptr(yl),
                   L.DTYPE_CODE[acc], slices, total, L.ptr(plan["sum_ptr"]), L.ptr(plan["sum_pair"]), L.ptr(part),
                   L.ptr(w), None, L.stream_ptr())
            outs.append(w.view(n_c, R).cpu().numpy())
        y = np.zeros((n, R))
        np.add.at(y, sub_idx, yl.double().cpu().numpy().reshape(slices, total, R).sum(0))
        ref = AR @ y
        assert np.abs(outs[0] - ref).max() <= 1e-13 * np.abs(ref).max()
        assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("prec", ["f64", "bf16"])
@pytest.mark.parametrize("R", [4, 16, 64])
def test_sub_restriction_preconditioner_matches(cuda, prec, R):
    """Hybrid Schwarz with R >= 2: the per-subdomain restriction (the default)
    gives the preconditioned vector of the y-first path up to rounding
    (SIMT and tensor-core local applies, overlapping Q1 subdomains)."""
    import dd_solvers_b200 as dd

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(2, 48, 6)
    pc = dd.HybridSchwarz(torch.float64, dd.Inv(DT[prec]), dd.CUDSS())
    pc.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0)
    r = torch.randn(A.shape[0], R, dtype=torch.float64, device=cuda)
    z1 = pc.solve(r)[0]
    assert pc._slices() in pc._subr  # the per-subdomain plan for the apply's ylocal slices
    pc.sub_restriction = False
    pc.mapped_restriction = False
    z0 = pc.solve(r)[0]
    err = ((z1 - z0).norm(dim=0) / z0.norm(dim=0)).max().item()
    assert err <= 1e-12, err


# ---------------------------------------------------------------------------
# Schwarz local apply / combine vs the oracle restatement
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("prec", ["f64", "f32", "bf16", "f16"])
@pytest.mark.parametrize("case", ["q1_2d", "q1_3d_uneven", "p1_rcb"])
def test_schwarz_apply(cuda, prec, case):
    import dd_solvers_b200 as dd
    from oracle import restatement as orc

    if case == "q1_2d":
        P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(2, 32, 4)
    elif case == "q1_3d_uneven":
        P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(3, 12, 3, kappa_seed=2, coarse="q1")
    else:
        P, A, owner, nparts, sub_ptr, sub_idx, R0 = p1_case(34, 8)
    At = torch_csr(A, cuda)
    for kind in ("additive", "hybrid"):
        cls = dd.AdditiveSchwarz if kind == "additive" else dd.HybridSchwarz
        pc = cls(torch.float64, dd.Inv(DT[prec]), dd.CUDSS())
        pc.setup(At, subdomains=(sub_ptr, sub_idx), coarse_restriction=R0)
        # oracle with the GPU's own (dequantised) blocks: isolates the apply
        blocks = [pc.store.block(i).cpu().numpy() for i in range(pc.n_solvers)]
        M = orc.Schwarz(A, sub_ptr, sub_idx, R0, block_dtype="f64", inverse_blocks=blocks)
        rng = np.random.default_rng(7)
        r = rng.standard_normal(A.shape[0])
        z = pc.solve(torch.as_tensor(r, device=cuda))[0].cpu().numpy()
        zr = M.additive(r) if kind == "additive" else M.hybrid(r)
        tol = 1e-12 if prec == "f64" else 2e-6
        assert np.linalg.norm(z - zr) <= tol * np.linalg.norm(zr), (kind, np.linalg.norm(z - zr) / np.linalg.norm(zr))


@pytest.mark.parametrize("layout", ["sym", "colmajor"])
@pytest.mark.parametrize("prec", ["f64", "f32", "bf16", "f16"])
def test_simt_apply_every_tuning_candidate(cuda, prec, layout):
    """Every configuration the autotuner may pick, for both block layouts, on
    subdomains of up to 34^2 = 1156 DOFs (full blocks, FP64: 5 row groups per
    thread, instantiated as 8; tiles: 37 tile rows, 703 tiles per block)."""
    import dd_solvers_b200 as dd
    from oracle import restatement as orc

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(2, 96, 3)
    pc = dd.AdditiveSchwarz(torch.float64, dd.Inv(DT[prec]), None)
    pc.symmetric_blocks = layout == "sym"
    pc.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx))
    assert pc.store.layout == layout
    blocks = [pc.store.block(i).cpu().numpy() for i in range(pc.n_solvers)]
    r = np.random.default_rng(5).standard_normal(A.shape[0])
    rt = torch.as_tensor(r, device=cuda)
    ref = np.concatenate([blocks[i] @ r[sub_idx[sub_ptr[i]:sub_ptr[i + 1]]] for i in range(pc.n_solvers)])
    tol = 1e-12 if prec in ("f64", "f32") else 2e-6
    for groups, kb in pc.tune_candidates:
        s = pc.scratch(1)
        try:
            pc._simt_apply(rt, s["ylocal"], 1, None, groups, kb)
        except Exception as e:  # a shape that needs more shared memory than a CTA has is refused
            assert "shared memory" in str(e), e
            continue
        parts = pc.parts if layout == "sym" else 1  # the split apply writes one ylocal slice per part
        got = s["ylocal"][: parts * len(sub_idx)].view(parts, -1).double().sum(0).cpu().numpy()
        assert np.linalg.norm(got - ref) <= tol * np.linalg.norm(ref), (groups, kb)
    from dd_solvers_b200 import _lib

    assert _lib.device_error() == 0


@pytest.mark.parametrize("lanes", [4, 8, 16, 32])
def test_spmv_csr_lanes(cuda, lanes):
    """Sub-warp CSR SpMV (coarse restriction): rows of 0..90 entries, a row
    count that is not a multiple of the rows per warp."""
    from dd_solvers_b200 import _lib as L

    rng = np.random.default_rng(lanes)
    n_rows, n_cols = 3001, 5000
    lens = rng.integers(0, 91, n_rows)
    crow = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    col = rng.integers(0, n_cols, int(crow[-1])).astype(np.int32)
    val = rng.standard_normal(int(crow[-1]))
    x = rng.standard_normal(n_cols)
    ref = sps.csr_matrix((val, col, crow), shape=(n_rows, n_cols)) @ x
    t = lambda a: torch.as_tensor(a, device=cuda)  # noqa: E731
    y = torch.full((n_rows,), np.nan, dtype=torch.float64, device=cuda)
    crow_t, col_t, val_t, x_t = t(crow), t(col), t(val), t(x)
    L.call("ddx_spmv_csr_lanes_f64", n_rows, lanes, L.ptr(crow_t), L.ptr(col_t), L.ptr(val_t), L.ptr(x_t),
           L.ptr(y), L.stream_ptr())
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("prec", ["f64", "f32", "bf16", "f16"])
@pytest.mark.parametrize("shape", ["equal", "uneven"])
@pytest.mark.parametrize("R", [1, 3])
def test_small_subdomain_apply(cuda, prec, shape, R):
    """The one-thread-per-entry kernel: equal contiguous blocks of 12 DOFs (the
    reference's DG layout, k_equal path) and overlapping subdomains of uneven
    size (binary search path), against the FP64 product of the stored blocks."""
    import dd_solvers_b200 as dd
    from dd_solvers_b200 import problems

    if shape == "equal":
        P = problems.q1_grid(2, 48)
        A = P.matrix
        n = A.shape[0]
        k = 12
        m = n // k
        A = A[: m * k][:, : m * k].tocsr()
        sub_ptr = np.arange(m + 1, dtype=np.int64) * k
        sub_idx = np.arange(m * k, dtype=np.int32)
    else:
        P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(2, 24, 6)
    pc = dd.AdditiveSchwarz(torch.float64, dd.Inv(DT[prec]), None)
    pc.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx))
    assert pc.store.layout == "colmajor" and pc.kmax <= pc.SMALL_KMAX
    assert (pc.k_equal > 0) == (shape == "equal")
    assert (pc.SMALL, 0) in pc.tune_candidates
    blocks = [pc.store.block(i).cpu().numpy() for i in range(pc.n_solvers)]
    r = np.random.default_rng(7).standard_normal((A.shape[0], R))
    ref = np.concatenate([blocks[i] @ r[sub_idx[sub_ptr[i]:sub_ptr[i + 1]]] for i in range(pc.n_solvers)])
    s = pc.scratch(R)
    pc._simt_apply(torch.as_tensor(r, device=cuda).reshape(-1), s["ylocal"], R, None, pc.SMALL, 0)
    got = s["ylocal"][: len(sub_idx) * R].double().view(-1, R).cpu().numpy()
    tol = 1e-13 if prec == "f64" else (1e-12 if prec == "f32" and pc.acc_dtype == torch.float64 else 2e-6)
    assert np.linalg.norm(got - ref) <= tol * np.linalg.norm(ref)


@pytest.mark.parametrize("prec", ["f32", "bf16", "f16"])
def test_block_quantisation_matches_oracle(cuda, prec):
    """Stored blocks equal the oracle's power-of-two-scaled rounding of the FP64 inverse."""
    import dd_solvers_b200 as dd
    from oracle import restatement as orc

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(2, 24, 3)
    pc = dd.AdditiveSchwarz(torch.float64, dd.Inv(DT[prec]), dd.CUDSS())
    pc.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0)
    pc64 = dd.AdditiveSchwarz(torch.float64, dd.Inv(), dd.CUDSS())
    pc64.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0)
    for i in range(pc.n_solvers):
        if i in pc.store.shifted:  # re-rounded with a shift to stay positive definite
            assert float(torch.linalg.eigvalsh(pc.store.block(i)).min()) > 0
            continue
        inv64 = pc64.store.block(i).cpu().numpy()
        s, Q = orc.quantize(inv64, prec)
        assert float(pc.store.scale[i]) == s
        assert np.array_equal(pc.store.block(i).cpu().numpy(), s * Q)


def test_local_apply_multi_rhs_matches_columns(cuda):
    import dd_solvers_b200 as dd

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(2, 32, 4)
    pc = dd.HybridSchwarz(torch.float64, dd.Inv(torch.bfloat16), dd.CUDSS())
    pc.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0)
    r = torch.randn(A.shape[0], 8, dtype=torch.float64, device=cuda)
    Z = pc.solve(r)[0]
    for j in range(8):
        zj = pc.solve(r[:, j].contiguous())[0]
        assert torch.allclose(Z[:, j], zj, rtol=0, atol=1e-14 * float(zj.abs().max()))


@pytest.mark.parametrize("R", [2, 16, 64])
@pytest.mark.parametrize("kind", ["additive", "hybrid"])
def test_schwarz_apply_multi_rhs_matches_oracle(cuda, R, kind):
    """(n, R) blocks of right-hand sides through the column-pair combine kernel and the
    grouped coarse GEMV, FP64 blocks: every column equals the oracle's apply."""
    import dd_solvers_b200 as dd
    from oracle import restatement as orc

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(3, 12, 3, kappa_seed=2, coarse="q1")
    cls = dd.AdditiveSchwarz if kind == "additive" else dd.HybridSchwarz
    pc = cls(torch.float64, dd.Inv(), dd.CUDSS())
    pc.setup(torch_csr(A, cuda), subdomains=(sub_ptr, sub_idx), coarse_restriction=R0)
    M = orc.Schwarz(A, sub_ptr, sub_idx, R0)
    r = np.random.default_rng(R).standard_normal((A.shape[0], R))
    Z = pc.solve(torch.as_tensor(r, device=cuda))[0].cpu().numpy()
    Zr = M.additive(r) if kind == "additive" else M.hybrid(r)
    err = np.linalg.norm(Z - Zr, axis=0) / np.linalg.norm(Zr, axis=0)
    assert err.max() <= 1e-12, err.max()


@pytest.mark.parametrize("R", [1, 2, 4, 8, 16, 32, 64])
@pytest.mark.parametrize("n_c", [1, 33, 257, 1000])
def test_coarse_gemv_matches_matmul(cuda, R, n_c):
    from dd_solvers_b200 import _lib as L

    g = torch.Generator(device=cuda).manual_seed(R * 1000 + n_c)
    Ainv = torch.randn(n_c, n_c, dtype=torch.float64, device=cuda, generator=g)
    w = torch.randn(n_c, R, dtype=torch.float64, device=cuda, generator=g)
    yc = torch.full((n_c, R), float("nan"), dtype=torch.float64, device=cuda)
    L.call("ddx_coarse_gemv_f64", n_c, R, L.ptr(Ainv), L.ptr(w), L.ptr(yc), None, L.stream_ptr())
    ref = Ainv @ w
    assert torch.allclose(yc, ref, rtol=1e-12, atol=1e-12 * float(ref.abs().max()))


@pytest.mark.parametrize("R", [16, 32, 64])
@pytest.mark.parametrize("n_c", [1, 33, 257, 1000, 3375])
def test_coarse_gemm_matches_matmul(cuda, R, n_c):
    """Tiled coarse GEMM with and without a split of Ainv's columns (scratch),
    against torch's FP64 product; a repeated call gives the same bits."""
    from dd_solvers_b200 import _lib as L

    g = torch.Generator(device=cuda).manual_seed(R * 7 + n_c)
    Ainv = torch.randn(n_c, n_c, dtype=torch.float64, device=cuda, generator=g)
    w = torch.randn(n_c, R, dtype=torch.float64, device=cuda, generator=g)
    ref = Ainv @ w
    scratch = torch.empty(16 * n_c * R, dtype=torch.float64, device=cuda)
    for sc, n_sc in ((None, 0), (scratch, scratch.numel())):
        outs = []
        for _ in range(2):
            yc = torch.full((n_c, R), float("nan"), dtype=torch.float64, device=cuda)
            L.call("ddx_coarse_gemm_f64", n_c, R, L.ptr(Ainv), L.ptr(w), L.ptr(yc), L.ptr(sc), n_sc, None,
                   L.stream_ptr())
            outs.append(yc)
        assert torch.allclose(outs[0], ref, rtol=1e-12, atol=1e-12 * float(ref.abs().max()))
        assert torch.equal(outs[0], outs[1])


@pytest.mark.parametrize("prec", ["f64", "f32", "bf16", "f16"])
def test_symmetric_tiles_apply_matches_fp64_product(cuda, prec):
    """Upper-triangle-tile apply on uneven RCB subdomains (k not a multiple of
    32) against the FP64 product of the same stored blocks; the stored blocks
    are exactly symmetric and within rounding of the full-layout blocks."""
    import dd_solvers_b200 as dd

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = p1_case(60, 4)
    At = torch_csr(A, cuda)
    pc = dd.AdditiveSchwarz(torch.float64, dd.Inv(DT[prec]), None)
    pc.setup(At, subdomains=(sub_ptr, sub_idx))
    assert pc.store.layout == "sym"
    full = dd.AdditiveSchwarz(torch.float64, dd.Inv(DT[prec]), None)
    full.symmetric_blocks = False
    full.setup(At, subdomains=(sub_ptr, sub_idx))
    r = np.random.default_rng(3).standard_normal(A.shape[0])
    y = pc._local_sum(torch.as_tensor(r, device=cuda), 1)[:, 0].cpu().numpy()
    num = den = 0.0
    for i in range(pc.n_solvers):
        Bi = pc.store.block(i)
        assert torch.equal(Bi, Bi.T)
        Fi = full.store.block(i)
        if i in pc.store.shifted:  # its plain 16-bit rounding was indefinite: re-rounded with a shift
            assert float(torch.linalg.eigvalsh(Bi).min()) > 0
        else:
            assert torch.allclose(Bi, Fi, rtol=0, atol=float(Fi.abs().max()) * (1e-12 if prec == "f64" else 1e-2))
        idx = sub_idx[sub_ptr[i]:sub_ptr[i + 1]]
        ref = Bi.cpu().numpy() @ r[idx]
        num += np.linalg.norm(y[sub_ptr[i]:sub_ptr[i + 1]] - ref) ** 2
        den += np.linalg.norm(ref) ** 2
    tol = 1e-12 if prec in ("f64", "f32") else 2e-6
    assert (num / den) ** 0.5 <= tol, (num / den) ** 0.5
    from dd_solvers_b200 import _lib

    assert _lib.device_error() == 0


def test_bsr_dg_pattern(cuda):
    """DG triangle block structure (P2, 6 DOFs per element) with uneven rows (2-4 blocks)."""
    from dd_solvers_b200 import FastBSR, problems

    crow, col = problems.dg_bsr_pattern_2d(9)
    bs = problems.dg_block_size(2, 2)
    nbr = len(crow) - 1
    vals = torch.randn(int(crow[-1]), bs, bs, dtype=torch.float64, generator=torch.Generator().manual_seed(1))
    m = torch.sparse_bsr_tensor(torch.as_tensor(crow.astype(np.int64)), torch.as_tensor(col.astype(np.int64)), vals,
                                size=(nbr * bs, nbr * bs))
    x = torch.randn(nbr * bs, dtype=torch.float64)
    expected = (m.to_dense() @ x).to(cuda)
    y = FastBSR(m.to(cuda)) @ x.to(cuda)
    assert torch.allclose(y, expected, rtol=1e-12, atol=1e-12)


def test_bsr_dg_pattern_3d(cuda):
    """DG tetrahedron block structure (P2, 10 DOFs per element, 3-5 blocks per row)."""
    from dd_solvers_b200 import FastBSR, problems

    crow, col = problems.dg_bsr_pattern_3d(3)
    bs = problems.dg_block_size(3, 2)
    nbr = len(crow) - 1
    vals = torch.randn(int(crow[-1]), bs, bs, dtype=torch.float64, generator=torch.Generator().manual_seed(2))
    m = torch.sparse_bsr_tensor(torch.as_tensor(crow.astype(np.int64)), torch.as_tensor(col.astype(np.int64)), vals,
                                size=(nbr * bs, nbr * bs))
    x = torch.randn(nbr * bs, dtype=torch.float64)
    expected = (m.to_dense() @ x).to(cuda)
    y = FastBSR(m.to(cuda)) @ x.to(cuda)
    assert torch.allclose(y, expected, rtol=1e-12, atol=1e-12)


def test_device_partitioning_on_gpu(cuda):
    """RCB owners and overlapping subdomains computed on the GPU equal the host
    versions (C5-style jittered P1 nodes, 256 parts, one layer of overlap)."""
    from dd_solvers_b200 import partition, problems

    P = problems.p1_jittered(257, 0.3, 1.0, 11)
    o_host = partition.rcb_owner(P.coords, 256)
    o_dev = partition.rcb_owner_device(torch.as_tensor(P.coords, device=cuda), 256)
    assert np.array_equal(o_host, o_dev.cpu().numpy())
    sp, si = partition.overlapping_subdomains(P.matrix, o_host, 256, 1)
    sp_t, si_t = partition.overlapping_subdomains_device(
        torch.as_tensor(P.matrix.indptr, device=cuda), torch.as_tensor(P.matrix.indices, device=cuda), o_dev, 256, 1)
    assert np.array_equal(sp, sp_t.cpu().numpy()) and np.array_equal(si, si_t.cpu().numpy())
