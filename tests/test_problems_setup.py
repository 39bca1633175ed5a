"""Host-side logic on CPU: assemblers, partitions, coarse spaces, setup layouts, C ABI."""
import ctypes
import itertools
import os
import re

import numpy as np
import pytest
import scipy.sparse as sps
import torch

from dd_solvers_b200 import partition, problems
from dd_solvers_b200 import setup_ops as so
from helpers import p1_case, q1_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _q1_brute(dim, n_el, kappa):
    h = 1.0 / n_el
    K = problems.q1_reference_stiffness(dim) * h ** (dim - 2)
    m = n_el - 1
    rows, cols, vals = [], [], []
    for c in itertools.product(range(n_el), repeat=dim):
        nodes = []
        for a in range(2 ** dim):
            bits = [(a >> d) & 1 for d in range(dim)]
            nodes.append([c[dim - 1 - d] + bits[d] for d in range(dim)])
        for a in range(2 ** dim):
            for b in range(2 ** dim):
                pa, pb = nodes[a], nodes[b]
                if any(q == 0 or q == n_el for q in pa + pb):
                    continue
                la = lb = 0
                for d in reversed(range(dim)):
                    la = la * m + pa[d] - 1
                    lb = lb * m + pb[d] - 1
                rows.append(la)
                cols.append(lb)
                vals.append(kappa[c] * K[a, b])
    return sps.csr_matrix((vals, (rows, cols)), shape=(m ** dim, m ** dim))


@pytest.mark.parametrize("dim,n_el", [(2, 6), (3, 4)])
def test_q1_stencil_assembly_matches_element_loop(dim, n_el):
    kappa = np.exp(np.random.default_rng(dim).standard_normal((n_el,) * dim))
    A = problems.q1_grid(dim, n_el, kappa).matrix
    B = _q1_brute(dim, n_el, kappa)
    assert abs(A - B).max() < 1e-14
    assert A.has_sorted_indices
    assert np.linalg.eigvalsh(A.toarray()).min() > 0


def test_p1_jittered_spd_and_consistent():
    P = problems.p1_jittered(9, 0.3, 1.0, 0)
    A = P.matrix.toarray()
    assert np.allclose(A, A.T)
    assert np.linalg.eigvalsh(A).min() > 0
    # constant coefficient, no jitter: the 5-point Laplacian (diagonal pair cancels)
    P0 = problems.p1_jittered(6, 0.0, 0.0, 0)
    A0 = P0.matrix.toarray()
    assert np.allclose(np.diag(A0), 4.0)
    assert np.allclose(A0[0, 1], -1.0) and np.allclose(A0[0, 5], 0.0)


def test_grf_statistics():
    g = problems.gaussian_random_field(64, 0.1, seed=0)
    assert g.shape == (64, 64)
    assert 0.3 < g.std() < 2.0
    g2 = problems.gaussian_random_field(64, 0.1, seed=0)
    assert np.array_equal(g, g2)


def test_box_partition_sizes():
    owner, n = partition.box_owner((255, 255), 8)
    c = np.bincount(owner, minlength=n)
    assert n == 64 and c.min() >= 31 * 31 and c.max() == 32 * 32
    owner3, n3 = partition.box_owner((127,) * 3, 16)
    c3 = np.bincount(owner3, minlength=n3)
    assert n3 == 4096 and c3.max() == 512


def test_overlap_and_transpose_map():
    P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(2, 16, 4)
    ks = np.diff(sub_ptr)
    assert ks.max() == 6 * 6  # 4x4 owned + one layer on each side
    for i in range(nparts):
        idx = sub_idx[sub_ptr[i]:sub_ptr[i + 1]]
        assert np.all(np.diff(idx) > 0)
        assert set(np.flatnonzero(owner == i)) <= set(idx)
    dof_ptr, dof_src = so.transpose_map(torch.as_tensor(sub_idx), A.shape[0])
    dof_ptr, dof_src = dof_ptr.numpy(), dof_src.numpy()
    for d in range(A.shape[0]):
        pos = dof_src[dof_ptr[d]:dof_ptr[d + 1]]
        assert np.all(sub_idx[pos] == d) and np.all(np.diff(pos) > 0)
    assert dof_ptr[-1] == len(sub_idx)


def test_rcb_uneven_partition():
    # 66 interior nodes per axis: the second bisection level splits 33 node
    # lines at the middle line, where jitter decides the side
    P = problems.p1_jittered(68, 0.3, 1.0, 1)
    owner = partition.rcb_owner(P.coords, 16)
    c = np.bincount(owner, minlength=16)
    assert c.sum() == P.matrix.shape[0] and c.min() > 0 and c.max() != c.min()


def test_q1_coarse_restriction_partition_of_unity():
    R = partition.q1_coarse_restriction(2, 16, 4)
    assert R.shape == (9, 225)
    # interior fine nodes far from the boundary are interpolated with weights summing to 1
    s = np.asarray(R.sum(axis=0)).ravel().reshape(15, 15)
    assert np.allclose(s[3:12, 3:12], 1.0)
    R3 = partition.q1_coarse_restriction(3, 8, 2)
    assert R3.shape == (1, 343) and np.isclose(R3.max(), 1.0)


def test_sell32_roundtrip():
    A = p1_case(20, 4)[1]
    crow = torch.as_tensor(A.indptr.astype(np.int64))
    sp, sw, sc, sv = so.csr_to_sell32(crow, torch.as_tensor(A.indices.astype(np.int64)), torch.as_tensor(A.data))
    n = A.shape[0]
    D = np.zeros((n, n))
    sp, sw, sc, sv = sp.numpy(), sw.numpy(), sc.numpy(), sv.numpy()
    for s in range(len(sw)):
        for l in range(32):
            r = 32 * s + l
            if r >= n:
                continue
            for j in range(sw[s]):
                D[r, sc[sp[s] + 32 * j + l]] += sv[sp[s] + 32 * j + l]
    assert np.array_equal(D, A.toarray())


@pytest.mark.parametrize("shuffled", [False, True])
def test_extract_blocks_matches_scipy(shuffled):
    """Blocks A[idx][:, idx] for ascending index lists and for lists in any
    order (a sharded rank's local numbering)."""
    P, A, owner, nparts, sub_ptr, sub_idx, R0 = p1_case(20, 4)
    if shuffled:
        rng = np.random.default_rng(3)
        sub_idx = sub_idx.copy()
        for i in range(nparts):
            rng.shuffle(sub_idx[sub_ptr[i]:sub_ptr[i + 1]])
    crow = torch.as_tensor(A.indptr.astype(np.int64))
    col = torch.as_tensor(A.indices.astype(np.int64))
    val = torch.as_tensor(A.data)
    ks = np.diff(sub_ptr)
    kpad = so.round_up(int(ks.max()), 16)
    blk = so.extract_blocks(crow, col, val, torch.as_tensor(sub_ptr), torch.as_tensor(sub_idx), 0, nparts, kpad)
    for i in range(nparts):
        idx = sub_idx[sub_ptr[i]:sub_ptr[i + 1]]
        k = len(idx)
        assert np.array_equal(blk[i, :k, :k].numpy(), A[idx][:, idx].toarray())
        assert np.array_equal(blk[i, k:, k:].numpy(), np.eye(kpad - k))


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32, torch.bfloat16, torch.float16])
def test_blockstore_layout_and_quantisation(dtype):
    from oracle import restatement as orc

    ks = np.array([5, 12, 0, 9])
    store = so.BlockStore(ks, dtype, "cpu")
    kpad = 16
    rng = np.random.default_rng(0)
    inv = torch.zeros(4, kpad, kpad, dtype=torch.float64)
    for i, k in enumerate(ks):
        inv[i, :k, :k] = torch.as_tensor(rng.standard_normal((k, k)) * 1e-3)
    store.put(0, inv)
    name = {torch.float64: "f64", torch.float32: "f32", torch.bfloat16: "bf16", torch.float16: "f16"}[dtype]
    V = 16 // so.ELEM_BYTES[dtype]
    for i, k in enumerate(ks):
        assert int(store.blk_off[i]) * so.ELEM_BYTES[dtype] % 16 == 0
        if k == 0:
            continue
        s, Q = orc.quantize(inv[i, :k, :k].numpy(), name)
        assert np.array_equal(store.block(i).numpy(), s * Q)
        # column-major with ld = round_up(k, V) and zero padding rows
        ld = (k + V - 1) // V * V
        raw = store.data[store.off_np[i]:store.off_np[i] + k * ld].view(k, ld)
        assert torch.all(raw[:, k:] == 0)


def test_capi_exports_every_declared_symbol():
    """libddx.so loads here (no GPU) and exports exactly what include/ddx.h declares."""
    import ctypes

    from dd_solvers_b200 import _lib

    hdr = open(os.path.join(ROOT, "include", "ddx.h")).read()
    declared = set(re.findall(r"^\w[\w\s\*]*?\b(ddx_\w+)\s*\(", hdr, flags=re.M))
    assert declared, "no declarations found"
    lib = _lib.lib()
    for name in declared:
        assert hasattr(lib, name), name
    assert declared == set(_lib.exported_symbols()) | (declared - set(_lib.exported_symbols()))
    assert set(_lib.exported_symbols()) <= declared


def test_capi_argument_checks_without_gpu():
    from dd_solvers_b200 import _lib

    lib = _lib.lib()
    assert lib.ddx_pcg_reset(3, None, None, 10, 0, 1e-8, 0.0, None) == 1
    assert b"unsupported R=3" in lib.ddx_last_error()
    assert lib.ddx_gemv_strided_batched(1, 3, None, 0, None, None, 1, None) == 1
    assert b"Double-Float" in lib.ddx_last_error() or b"null" in lib.ddx_last_error()
    assert lib.ddx_spmv_sell_f64(100, 3, None, None, None, None, None, None, None, 0, None, None, None, None,
                                 None, None) == 1
    assert lib.ddx_partials_len(64) == 592 * 4 * 64
    # the deferred-reduction epilogue checks its arguments before any launch
    assert lib.ddx_pcg_finalize(3, _lib.FIN_RR, None, None, None, None) == 1
    assert lib.ddx_pcg_finalize(4, _lib.FIN_RR, None, None, None, None) == 1
    assert b"null state" in lib.ddx_last_error()
    one = ctypes.c_double(0.0)
    flag = ctypes.c_int(0)
    assert lib.ddx_pcg_finalize(4, 9, ctypes.byref(one), ctypes.byref(flag), ctypes.byref(one), None) == 1
    assert b"unknown kind 9" in lib.ddx_last_error()
    # the epilogue after a BSR product: y, a PCG mode and the state are required, checked before any launch
    assert lib.ddx_spmv_epilogue_f64(10, None, None, None, 1, None, None, None, None, None, None) == 1
    assert b"bad arguments" in lib.ddx_last_error()
    y = ctypes.byref(one)
    assert lib.ddx_spmv_epilogue_f64(10, y, y, None, 0, None, None, None, None, None, None) == 1
    assert b"bad mode 0" in lib.ddx_last_error()
    assert lib.ddx_spmv_epilogue_f64(10, y, y, None, 1, None, None, None, None, None, None) == 1
    assert b"needs state" in lib.ddx_last_error()
    st = (ctypes.byref(one), ctypes.byref(flag), ctypes.byref(one), ctypes.byref(one), ctypes.byref(flag))
    assert lib.ddx_spmv_epilogue_f64(10, y, y, None, 2, *st, None) == 1
    assert b"residual mode needs b" in lib.ddx_last_error()
    # the BSR kernel's block sizes end where the PCG's BSR form stops being used
    from dd_solvers_b200.solvers import BSR_MAX_BLOCK
    rp = ctypes.byref(flag)
    assert lib.ddx_spmv_bsr(1, BSR_MAX_BLOCK + 1, rp, rp, y, y, y, _lib.F64, None) != 0
    assert f"block size {BSR_MAX_BLOCK + 1} not in 1..{BSR_MAX_BLOCK}".encode() in lib.ddx_last_error()


def test_solver_rejects_cpu_tensors():
    import dd_solvers_b200 as dd
    from dd_solvers_b200 import _lib

    A = torch.eye(3, dtype=torch.float64).to_sparse_csr()
    with pytest.raises(_lib.DDXError):
        dd.CG(bsr_matmul=False).setup(A)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32, torch.bfloat16, torch.float16])
def test_blockstore_symmetric_tiles(dtype):
    """Upper-triangle tile layout: round trip equals the full layout of the
    symmetrised blocks, and each element sits where the kernel reads it."""
    ks = np.array([5, 40, 0, 70, 64])
    rng = np.random.default_rng(1)
    inv = torch.zeros(len(ks), 80, 80, dtype=torch.float64)
    for i, k in enumerate(ks):
        m = rng.standard_normal((k, k))
        inv[i, :k, :k] = torch.as_tensor(m + 0.3 * m.T) * 1e-3  # not symmetric: put symmetrises
    sym = so.BlockStore(ks, dtype, "cpu", layout="sym")
    sym.put(0, inv)
    full = so.BlockStore(ks, dtype, "cpu")
    full.put(0, 0.5 * (inv + inv.transpose(1, 2)))
    V = 16 // so.ELEM_BYTES[dtype]
    for i, k in enumerate(ks):
        if k == 0:
            continue
        assert torch.equal(sym.block(i), full.block(i))
        Q = sym.dense_q(i)
        nt = (k + 31) // 32
        tau = 0
        for I in range(nt):
            for J in range(I, nt):
                base = int(sym.off_np[i]) + tau * 1024
                for r, c in ((0, 0), (1, 9), (7, 31), (30, 17)):
                    sw = ((r >> 1) & 3) if so.ELEM_BYTES[dtype] == 2 else (r & 7)
                    pos = base + r * 32 + (((c // V) ^ sw) * V) + c % V
                    gr, gc = I * 32 + r, J * 32 + c
                    want = Q[gr, gc] if gr < k and gc < k else 0
                    assert sym.data[pos] == want, (i, I, J, r, c)
                tau += 1
        assert int(sym.off_np[i + 1]) - int(sym.off_np[i]) == tau * 1024


def test_umma_symmetric_tile_layout():
    """Upper-triangle 128 x 128 tensor-core tiles: every element where the kernel reads it."""
    ks = np.array([130, 0, 300])
    rng = np.random.default_rng(2)
    inv = torch.zeros(len(ks), 304, 304, dtype=torch.float64)
    for i, k in enumerate(ks):
        m = rng.standard_normal((k, k))
        inv[i, :k, :k] = torch.as_tensor(m + m.T)
    st = so.BlockStore(ks, torch.bfloat16, "cpu", layout="sym")
    st.put(0, inv)
    ut = so.UmmaSymTileStore(st)
    data = ut.data
    for i, k in enumerate(ks):
        if k == 0:
            continue
        Q = st.dense_q(i)
        nt = (k + 127) // 128
        base = int(ut.off_np[i])
        assert int(ut.tile_off[i]) == 2 * base
        tau = 0
        for I in range(nt):
            for J in range(I, nt):
                for r, c in ((0, 0), (5, 70), (127, 127), (64, 9), (3, 63)):
                    h, cc = divmod(c, 64)
                    pos = base + tau * 16384 + h * 8192 + r * 64 + ((cc // 8) ^ (r % 8)) * 8 + cc % 8
                    gr, gc = I * 128 + r, J * 128 + c
                    want = Q[gr, gc] if gr < k and gc < k else 0
                    assert data[pos] == want, (i, I, J, r, c)
                tau += 1
        assert int(ut.off_np[i + 1]) - base == tau * 16384


def test_dg_block_patterns_match_the_reference_meshes():
    """The synthetic DG block structures have the block counts of the reference's
    BSR-benchmark meshes (results/benchmark_bsrmv.csv: S8 2D and S5 3D)."""
    crow, col = problems.dg_bsr_pattern_2d(256)
    assert len(crow) - 1 == 131072 and crow[-1] == 523264
    crow3, col3 = problems.dg_bsr_pattern_3d(32)
    assert len(crow3) - 1 == 196608 and crow3[-1] == 970752
    n = len(crow3) - 1
    M = sps.csr_matrix((np.ones(len(col3)), col3, crow3), shape=(n, n))
    assert abs(M - M.T).nnz == 0 and np.diff(crow3).max() == 5


@pytest.mark.parametrize("parts", [8, 64])
def test_device_partitioning_matches_host(parts):
    """RCB owners and overlap growth in torch (here on CPU tensors; the GPU
    test runs them on cuda) equal the numpy/SciPy versions exactly."""
    import torch

    from dd_solvers_b200 import partition, problems

    P = problems.p1_jittered(97, 0.3, 1.0, 5)
    o_host = partition.rcb_owner(P.coords, parts)
    o_dev = partition.rcb_owner_device(torch.as_tensor(P.coords), parts).numpy()
    assert np.array_equal(o_host, o_dev)
    for overlap in (0, 1, 2):
        sp, si = partition.overlapping_subdomains(P.matrix, o_host, parts, overlap)
        sp_t, si_t = partition.overlapping_subdomains_device(
            torch.as_tensor(P.matrix.indptr), torch.as_tensor(P.matrix.indices), torch.as_tensor(o_host), parts,
            overlap)
        assert np.array_equal(sp, sp_t.numpy()) and np.array_equal(si, si_t.numpy())


@pytest.mark.parametrize("dim,n_el,parts", [(2, 12, 3), (2, 30, 5), (3, 18, 3), (3, 32, 4)])
def test_device_coarse_restrictions_match_host(dim, n_el, parts):
    """The Q1 and P0 coarse restrictions built in torch (CPU tensors here, cuda
    in the bench) equal the SciPy ones entry for entry, and the device CSR
    transpose the Schwarz setup uses equals SciPy's."""
    import torch

    from dd_solvers_b200 import partition
    from dd_solvers_b200 import solvers as S
    from dd_solvers_b200.setup_ops import scipy_csr

    a = partition.q1_coarse_restriction(dim, n_el, parts)
    b = scipy_csr(partition.q1_coarse_restriction_device(dim, n_el, parts, "cpu"))
    assert np.array_equal(a.indptr, b.indptr) and np.array_equal(a.indices, b.indices)
    assert np.array_equal(a.data, b.data)
    own = np.random.default_rng(dim * n_el).integers(0, parts * parts, (n_el - 1) ** dim)
    a0 = partition.p0_restriction(own, parts * parts)
    b0 = scipy_csr(partition.p0_restriction_device(torch.as_tensor(own), parts * parts))
    assert np.array_equal(a0.indptr, b0.indptr) and np.array_equal(a0.indices, b0.indices)
    assert np.array_equal(a0.data, b0.data)
    crow, col, val, n_c = S._restriction_dev(partition.q1_coarse_restriction_device(dim, n_el, parts, "cpu"),
                                             a.shape[1], "cpu")
    assert n_c == a.shape[0]
    pt_crow, pt_col, pt_val = S._transpose_dev(crow, col, val, n_c, a.shape[1])
    At = a.T.tocsr()
    At.sort_indices()
    assert np.array_equal(pt_crow.numpy(), At.indptr) and np.array_equal(pt_col.numpy(), At.indices)
    assert np.array_equal(pt_val.numpy(), At.data)


def test_spd_guard_keeps_rounded_blocks_positive_definite():
    """A block whose BF16 rounding is indefinite (inverse of cond ~1e6) is
    re-rounded with a diagonal shift and comes out positive definite; a
    well-conditioned block in the same batch is stored exactly as without the
    guard (same bits, same scale)."""
    rng = np.random.default_rng(0)
    k = 256
    Qm, _ = np.linalg.qr(rng.standard_normal((k, k)))
    bad = (Qm * np.geomspace(1e-6, 1.0, k)) @ Qm.T         # eigenvalues 1e-6 .. 1
    good = (Qm * np.geomspace(0.5, 1.0, k)) @ Qm.T
    inv = torch.as_tensor(np.stack([bad, good]))
    plain = so.BlockStore(np.array([k, k]), torch.bfloat16, "cpu", layout="sym")
    plain.spd_guard = False
    plain.put(0, inv.clone())
    assert np.linalg.eigvalsh(plain.block(0).numpy()).min() < 0  # the case the guard is for
    st = so.BlockStore(np.array([k, k]), torch.bfloat16, "cpu", layout="sym")
    st.put(0, inv.clone())
    assert list(st.shifted) == [0] and st.shifted[0] > 0
    assert np.linalg.eigvalsh(st.block(0).numpy()).min() > 0
    assert torch.equal(st.dense_q(1), plain.dense_q(1)) and float(st.scale[1]) == float(plain.scale[1])


def _entries(plan, p):
    """(slot, value) entries of ylocal row p in a restriction plan."""
    out = []
    for e in range(2):
        if int(plan["f_slot"][2 * p + e]) != 255:
            out.append((int(plan["f_slot"][2 * p + e]), float(plan["f_val"][2 * p + e])))
    for t in range(int(plan["ov_ptr"][p]), int(plan["ov_ptr"][p + 1])):
        out.append((int(plan["ov_slot"][t]), float(plan["ov_val"][t])))
    return out


def _restrict_with_plan(plan, sub_ptr, ylocal, n_c, R):
    """The two passes of ddx_schwarz_restrict_sub in numpy (any fixed order)."""
    S = plan["slices"]
    total = int(sub_ptr[-1])
    base, nsl = plan["slot_base"].numpy(), plan["n_slots"].numpy()
    partial = np.zeros((plan["n_pairs"], R))
    for i in range(len(sub_ptr) - 1):
        for sc in range(S):
            for p in range(sub_ptr[i] + sc * total, sub_ptr[i + 1] + sc * total):
                for sl, v in _entries(plan, p):
                    assert sl < nsl[i]
                    partial[base[i] + sl] += v * ylocal[p]
    sp, sq = plan["sum_ptr"].numpy(), plan["sum_pair"].numpy()
    return np.stack([partial[sq[sp[c]:sp[c + 1]]].sum(0) for c in range(n_c)])


@pytest.mark.parametrize("case", ["q1_2d_p0", "q1_3d_q1", "p1_rcb"])
def test_subdomain_restriction_plan(case):
    """The per-subdomain restriction plan (slots of the coarse rows each
    subdomain touches, per-position entries; built with torch on the CPU):
    the two passes reproduce A_R y with y = sum_i R_i^T ylocal_i, also with
    ylocal split into slices; slots ascending in the coarse row, each coarse
    row's pairs in ascending subdomain order, every nonzero of A_R R_i^T once."""
    if case == "q1_2d_p0":
        P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(2, 24, 4)
    elif case == "q1_3d_q1":
        P, A, owner, nparts, sub_ptr, sub_idx, R0 = q1_case(3, 8, 2, kappa_seed=1, coarse="q1")
    else:
        P, A, owner, nparts, sub_ptr, sub_idx, R0 = p1_case(30, 8)
    AR = sps.csr_matrix(R0 @ A)
    AR.sort_indices()
    n_c, n = AR.shape
    args = (torch.as_tensor(AR.indptr.astype(np.int64)), torch.as_tensor(AR.indices.astype(np.int32)),
            torch.as_tensor(AR.data), n_c, n, torch.as_tensor(sub_ptr), torch.as_tensor(sub_idx))
    plan = so.subdomain_restriction(*args)
    nsub = len(sub_ptr) - 1
    # slots: the coarse rows each subdomain touches, ascending; pairs per coarse row
    pairs = []
    for i in range(nsub):
        cs = np.unique(AR[:, sub_idx[sub_ptr[i]:sub_ptr[i + 1]]].nonzero()[0])
        assert plan["n_slots"][i] == len(cs) and plan["slot_base"][i] == len(pairs)
        pairs += [(i, c) for c in cs]
    assert plan["n_pairs"] == len(pairs) and plan["max_slots"] == int(plan["n_slots"].max())
    sp, sq = plan["sum_ptr"].numpy(), plan["sum_pair"].numpy()
    for c in range(n_c):
        subs = [pairs[q][0] for q in sq[sp[c]:sp[c + 1]]]
        assert all(pairs[q][1] == c for q in sq[sp[c]:sp[c + 1]]) and subs == sorted(subs)
    # per-position entries: the A_R values of the position's DOF, slots ascending
    for i in range(nsub):
        for p in range(sub_ptr[i], sub_ptr[i + 1]):
            ent = _entries(plan, p)
            sl = np.array([e[0] for e in ent], dtype=np.int64)
            assert (np.diff(sl) > 0).all()
            cs = [pairs[int(plan["slot_base"][i]) + k][1] for k in sl]
            np.testing.assert_array_equal(np.array([e[1] for e in ent]), AR[cs, sub_idx[p]].toarray().ravel())
    R = 3
    for S in (1, 3):
        pl = plan if S == 1 else so.subdomain_restriction(*args, slices=S)
        yl = np.random.default_rng(S).standard_normal((S * int(sub_ptr[-1]), R))
        w = _restrict_with_plan(pl, sub_ptr, yl, n_c, R)
        y = np.zeros((n, R))
        np.add.at(y, sub_idx, yl.reshape(S, -1, R).sum(0))
        ref = AR @ y
        assert np.abs(w - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("cluster", [1, 7, 64, 10_000])
def test_row_clusters(cluster):
    """ddx_row_clusters (host code of the library): a permutation of the rows,
    cut into clusters of exactly `cluster` rows (but the last), each ascending
    and, on a 3D grid, compact: a 64-row cluster's neighbourhood (distinct
    columns) is well below that of 64 consecutive rows."""
    from dd_solvers_b200 import _lib as L

    A = sps.csr_matrix(q1_case(3, 24, 2)[1])
    n = A.shape[0]
    ip = torch.as_tensor(A.indptr.astype(np.int64))
    ix = torch.as_tensor(A.indices.astype(np.int64))
    order = torch.empty(n, dtype=torch.int32)
    L.call("ddx_row_clusters", n, ip.data_ptr(), ix.data_ptr(), cluster, order.data_ptr())
    o = order.numpy()
    assert np.array_equal(np.sort(o), np.arange(n))
    for i in range(0, n, cluster):
        assert (np.diff(o[i:i + cluster]) > 0).all()
    if cluster == 64:
        nb = np.mean([len(np.unique(A[o[i:i + 64]].indices)) for i in range(0, n - 64, 64)])
        nat = np.mean([len(np.unique(A[i:i + 64].indices)) for i in range(0, n - 64, 64)])
        assert nb < 0.7 * nat, (nb, nat)
    # a column out of range is refused (the tensors stay referenced during the call)
    bad_ptr = torch.as_tensor(np.array([0, 1, 2], dtype=np.int64))
    bad_idx = torch.as_tensor([0, 5], dtype=torch.int64)
    bad_out = torch.empty(2, dtype=torch.int32)
    with pytest.raises(L.DDXError):
        L.call("ddx_row_clusters", 2, bad_ptr.data_ptr(), bad_idx.data_ptr(), 4, bad_out.data_ptr())
