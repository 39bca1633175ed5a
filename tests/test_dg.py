"""The DG-SIPG discretisation of the reference's experiments, pinned to its logs.

``tests/golden/dg_experiments.json`` holds the residual histories that the
reference logged for its own CG runs on the 2D uniform-mesh problems at P1, P3
and P5 (``results/experiment_precisions.csv``); the oracle run on this
package's assembly must reproduce them.
"""
import json
import math
import os
import sys

import numpy as np
import pytest
import scipy.sparse as sps
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from dd_solvers_b200 import dg, problems  # noqa: E402
from oracle import restatement as rs  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden", "dg_experiments.json")


def golden_rows():
    with open(GOLDEN) as fh:
        return json.load(fh)


def golden(fine, solvers, coarse, prefix):
    for r in golden_rows():
        if (r["fine"], r["solvers"], r["coarse"]) == (fine, solvers, coarse) and r["solver"].startswith(prefix):
            return r
    raise KeyError((fine, solvers, coarse, prefix))


def scipy_csr(A):
    return sps.csr_matrix((A.values().numpy(), A.col_indices().numpy(), A.crow_indices().numpy()),
                          shape=tuple(A.shape))


def test_s0_block_sums_match_reference_test():
    """``src/experiments/tests/test_discretization.py:8-27``: rho = 1, delta = 7
    on the two-triangle mesh."""
    s = dg.sipg_p1(dg.uniform_mesh_2d(0), dg.CONSTANT_COEFFICIENT_2D)
    A = s.matrix.to_dense().numpy()
    delta = 7.0
    assert A.shape == (6, 6)
    assert np.isclose(A[:3, :3].sum(), delta * 5 / 2)
    assert np.isclose(A[3:, :3].sum(), -delta / 2)
    assert np.isclose(A[3:, 3:].sum(), delta * 5 / 2)
    assert np.isclose(A[:3, 3:].sum(), -delta / 2)


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_s0_block_sums_at_every_degree(p):
    """The same test at degree p: with rho = 1 a cell's constant has no
    gradient, so a block sum is its penalty alone, delta p^2 times the jump
    weights: 2 boundary edges + half the shared one (5/2) on the diagonal
    blocks, -1/2 off them."""
    s = dg.sipg(dg.uniform_mesh_2d(0), dg.CONSTANT_COEFFICIENT_2D, degree=p)
    A = s.matrix.to_dense().numpy()
    nb = s.block_size
    dp2 = 7.0 * p * p
    assert A.shape == (2 * nb, 2 * nb)
    assert np.isclose(A[:nb, :nb].sum(), dp2 * 5 / 2)
    assert np.isclose(A[nb:, :nb].sum(), -dp2 / 2)
    assert np.isclose(A[nb:, nb:].sum(), dp2 * 5 / 2)
    assert np.isclose(A[:nb, nb:].sum(), -dp2 / 2)


@pytest.mark.parametrize("m", [1, 2, 3])
def test_matrix_symmetric_positive_definite(m):
    A = dg.sipg_p1(dg.uniform_mesh_2d(m)).matrix.to_dense().numpy()
    assert np.abs(A - A.T).max() < 1e-12 * np.abs(A).max()
    assert np.linalg.eigvalsh(A).min() > 0


@pytest.mark.parametrize("m", [1, 4])
def test_block_structure_matches_bsr_benchmark_pattern(m):
    """Cell c's block row holds c and its edge neighbours; the block count is
    that of the reference's 2D BSR benchmark meshes."""
    mesh = dg.uniform_mesh_2d(m)
    A = dg.sipg_p1(mesh).matrix
    n = mesh.n_cells
    assert n == 2 * 4 ** m
    crow, col = A.crow_indices(), A.col_indices()
    rows3 = crow[1::3][: n] - crow[0:-1:3][: n]  # entries of each cell's first row
    blocks = int(rows3.sum()) // 3
    _, bcol = problems.dg_bsr_pattern_2d(1 << m)
    assert blocks == len(bcol)
    # every row has sorted columns
    for r in range(0, 3 * n, max(1, 3 * n // 50)):
        c = col[crow[r]:crow[r + 1]]
        assert bool((c[1:] > c[:-1]).all())


def test_cell_mappings():
    """``src/experiments/tests/test_meshing.py:36-61``: S2 -> C2 by centroid,
    S2 -> S1 four children per parent, S1 -> S1 the identity."""
    mesh = dg.uniform_mesh_2d(2)
    mp = dg.cell_mapping(mesh, "C2")
    assert mp.shape == (32,)
    ctr = mesh.vertices[mesh.cells].mean(dim=1)
    qx, qy = mp % 4, mp // 4
    assert bool(((qx / 4 < ctr[:, 0]) & (ctr[:, 0] < (qx + 1) / 4)).all())
    assert bool(((qy / 4 < ctr[:, 1]) & (ctr[:, 1] < (qy + 1) / 4)).all())
    mp = dg.cell_mapping(mesh, "S1")
    assert torch.equal(torch.bincount(mp), torch.full((8,), 4))
    # children sit inside their parent
    m1 = dg.uniform_mesh_2d(1)
    par = m1.vertices[m1.cells][mp]  # (32, 3, 2)
    a, b, c = par[:, 0], par[:, 1], par[:, 2]
    v0, v1 = b - a, c - a
    d = ctr - a
    det = v0[:, 0] * v1[:, 1] - v0[:, 1] * v1[:, 0]
    l1 = (d[:, 0] * v1[:, 1] - d[:, 1] * v1[:, 0]) / det
    l2 = (v0[:, 0] * d[:, 1] - v0[:, 1] * d[:, 0]) / det
    assert bool(((l1 > 0) & (l2 > 0) & (l1 + l2 < 1)).all())
    assert torch.equal(dg.cell_mapping(m1, "S1"), torch.arange(8))


@pytest.fixture(scope="module")
def s10():
    return dg.sipg_p1(dg.uniform_mesh_2d(10))


def test_s10_size_and_load_norm_match_reference_log(s10):
    """The S10 system: the reference logged its size, nnz and (as the first
    additive-Schwarz residual norm, x0 = 0) the load-vector norm."""
    row = golden("S10", "S8", "S8", "CG(AdditiveSchwarz(torch.float64, Inv(), CUDSS")
    assert s10.load.shape[0] == row["dofs"]
    assert s10.matrix.values().shape[0] == row["nnz"]
    b = float(torch.linalg.norm(s10.load))
    assert math.isclose(b, row["residual_norms"][0], rel_tol=1e-13)


@pytest.mark.parametrize("kind", ["additive", "hybrid"])
def test_s10_oracle_residual_history_matches_reference_log(s10, kind):
    """Fine S10, subdomains and P0 coarse aggregates S8 (48 DOFs each,
    131,072 coarse DOFs), FP64: the first twelve residual norms of the
    reference's logged run, reproduced to 1e-10."""
    prefix = {"additive": "CG(AdditiveSchwarz(torch.float64, Inv(), CUDSS",
              "hybrid": "CG(HybridSchwarz(torch.float64, Inv(), CUDSS"}[kind]
    row = golden("S10", "S8", "S8", prefix)
    A = scipy_csr(s10.matrix)
    b = s10.load.numpy()
    n_sol = 2 * 4 ** 8
    P = rs.ContiguousSchwarz(A, 3 * 4 ** 2, np.ones(n_sol, dtype=np.int64))
    M = P.additive if kind == "additive" else P.hybrid
    T0 = P.T0 if kind == "hybrid" else None
    _, meta = rs.pcg(A, b, M=M, T0=T0, rtol=1e-9, maxiter=12, raise_on_fail=False)
    ours = np.array(meta["residual norms"])
    ref = np.array(row["residual_norms"][: len(ours)])
    assert len(ours) == 12
    np.testing.assert_allclose(ours, ref, rtol=1e-10)


@pytest.mark.parametrize("case", [dg.CONTINUOUS_COEFFICIENT_2D, dg.CONSTANT_COEFFICIENT_2D], ids=["continuous", "constant"])
def test_sipg_converges_at_second_order(case):
    """Direct solves on S3..S6: the L2 error against the exact solution of
    ``problems.py:31-74`` falls by ~4x per refinement (P1, h -> h/2)."""
    import scipy.sparse.linalg as spla

    errs = []
    for m in range(3, 7):
        mesh = dg.uniform_mesh_2d(m)
        s = dg.sipg_p1(mesh, case)
        u = spla.spsolve(scipy_csr(s.matrix).tocsc(), s.load.numpy())
        errs.append(dg.l2_error(mesh, u, case.solution))
    assert errs[0] < 0.5  # the reference's bound at S3 (tests/test_experiments.py:37-41)
    ratio = errs[-2] / errs[-1]
    assert 3.7 < ratio < 4.3, errs


# ---------------------------------------------------------------------------
# degrees p = 2..5 (the reference's P3 and P5 experiments)
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("m", [1, 3])
@pytest.mark.parametrize("case", [dg.CONTINUOUS_COEFFICIENT_2D, dg.CONSTANT_COEFFICIENT_2D], ids=["continuous", "constant"])
def test_quadrature_assembly_matches_p1_closed_form(m, case):
    """The degree-p assembly (nodal basis, exact quadrature) at p = 1 against
    the closed form that the S10 logs pin: same pattern, entries to rounding."""
    mesh = dg.uniform_mesh_2d(m)
    a, b = dg.sipg_p1(mesh, case), dg._sipg_quadrature(mesh, case, 1)
    assert torch.equal(a.matrix.crow_indices(), b.matrix.crow_indices())
    assert torch.equal(a.matrix.col_indices(), b.matrix.col_indices())
    va, vb = a.matrix.values(), b.matrix.values()
    assert float((va - vb).abs().max()) <= 1e-13 * float(va.abs().max())
    assert float((a.load - b.load).abs().max()) <= 1e-13 * float(a.load.abs().max())


def test_reference_nodes_layout():
    """Vertices first, then each edge's interior points at the GLL points
    (edge 0 from vertex 1 to 2, edge 1 from 0 to 2, edge 2 from 0 to 1), then
    the interior; equispaced for p <= 2, the P3 interior point at the
    centroid, and every node set invariant under the triangle's rotation."""
    for p in range(1, 6):
        P = dg.reference_nodes(p)
        nb = (p + 1) * (p + 2) // 2
        assert P.shape == (nb, 2)
        np.testing.assert_array_equal(P[:3], [[0, 0], [1, 0], [0, 1]])
        g = dg._gll_points(p)[1:-1]
        k = p - 1
        np.testing.assert_allclose(P[3:3 + k], np.stack([1 - g, g], 1), atol=1e-15)
        np.testing.assert_allclose(P[3 + k:3 + 2 * k], np.stack([0 * g, g], 1), atol=1e-15)
        np.testing.assert_allclose(P[3 + 2 * k:3 + 3 * k], np.stack([g, 0 * g], 1), atol=1e-15)
        # rotation (x, y) -> (y, 1 - x - y) maps the node set onto itself
        Q = np.stack([P[:, 1], 1 - P[:, 0] - P[:, 1]], 1)
        d = np.abs(Q[:, None, :] - P[None, :, :]).sum(-1).min(1)
        assert d.max() < 1e-14
    np.testing.assert_allclose(dg.reference_nodes(2), [[0, 0], [1, 0], [0, 1], [.5, .5], [0, .5], [.5, 0]])
    # GLL points in closed form: roots of P_3' at +-1/sqrt(5), of P_5' at +-sqrt(1/3 -+ 2 sqrt(7) / 21)
    np.testing.assert_allclose(dg._gll_points(3), [0, .5 - 5 ** .5 / 10, .5 + 5 ** .5 / 10, 1], atol=1e-15)
    r5 = sorted([-(1 / 3 + 2 * 7 ** .5 / 21) ** .5, -(1 / 3 - 2 * 7 ** .5 / 21) ** .5,
                 (1 / 3 - 2 * 7 ** .5 / 21) ** .5, (1 / 3 + 2 * 7 ** .5 / 21) ** .5])
    np.testing.assert_allclose(dg._gll_points(5)[1:-1], (1 + np.array(r5)) / 2, atol=1e-15)
    np.testing.assert_allclose(dg.reference_nodes(3)[-1], [1 / 3, 1 / 3], atol=1e-15)
    # the nodal basis is the identity on the nodes
    P = dg.reference_nodes(5)
    v, _, _ = dg.nodal_basis(5, P[:, 0], P[:, 1])
    np.testing.assert_allclose(v, np.eye(21), atol=1e-12)


@pytest.mark.parametrize("p", [2, 3, 4, 5])
def test_higher_degree_matrix_symmetric_positive_definite(p):
    A = dg.sipg(dg.uniform_mesh_2d(2), degree=p).matrix.to_dense().numpy()
    assert A.shape[0] == 32 * (p + 1) * (p + 2) // 2
    assert np.abs(A - A.T).max() < 1e-13 * np.abs(A).max()
    assert np.linalg.eigvalsh(A).min() > 0


@pytest.mark.parametrize("p,fine", [(3, "S9"), (5, "S8")])
def test_higher_degree_size_and_load_norm_match_reference_log(p, fine):
    """The reference's P3 (S9) and P5 (S8) systems: DOFs and nnz from the
    block structure, and the load-vector norm (its first additive-Schwarz
    residual norm, x0 = 0), which depends on where the nodes sit: GLL-warped
    nodes match to rounding, equispaced interior nodes would be 17% off at P5."""
    row = next(r for r in golden_rows() if r.get("p") == p and r["fine"] == fine
               and r["solver"].startswith("CG(AdditiveSchwarz(torch.float64, Inv(), CUDSS"))
    mesh = dg.uniform_mesh_2d(int(fine[1:]))
    nb = (p + 1) * (p + 2) // 2
    (c1, _, _, _), _ = dg._edge_tables(mesh)
    assert mesh.n_cells * nb == row["dofs"]
    assert (mesh.n_cells + 2 * c1.numel()) * nb * nb == row["nnz"]
    b = float(torch.linalg.norm(dg.load_vector(mesh, degree=p)))
    assert math.isclose(b, row["residual_norms"][0], rel_tol=1e-12)


@pytest.mark.parametrize("p,ratio", [(2, 8.0), (3, 16.0)])
def test_higher_degree_converges_at_order_p_plus_one(p, ratio):
    """Direct solves on S4..S6 (continuous coefficient): the L2 error falls by
    ~2^(p+1) per refinement."""
    import scipy.sparse.linalg as spla

    case = dg.CONTINUOUS_COEFFICIENT_2D
    errs = []
    for m in range(4, 7):
        mesh = dg.uniform_mesh_2d(m)
        s = dg.sipg(mesh, case, p)
        u = spla.spsolve(scipy_csr(s.matrix).tocsc(), s.load.numpy())
        errs.append(dg.l2_error_p(mesh, u, case.solution, p))
    r = errs[-2] / errs[-1]
    assert 0.93 * ratio < r < 1.07 * ratio, errs


def test_experiment_grouping_higher_degree():
    """DOFs grouped by (coarse, solver) cells for p = 3: every solver holds
    its cells' 10 DOFs each, in contiguous runs."""
    from dd_solvers_b200 import dg_experiments

    A, b, kw, perm = dg_experiments.build("S4", "S3", "S2", device="cpu", return_perm=True, degree=3)
    assert A.shape == (512 * 10, 512 * 10) and b.shape == (5120,)
    assert kw["block_size"] == 10 and kw["dofs_per_solver"] == 40
    assert int(kw["solvers_per_coarse"].sum()) == 128
    assert torch.equal(torch.sort(perm).values, torch.arange(5120))
    cell = perm // 10
    f2s = dg.cell_mapping(dg.uniform_mesh_2d(4), "S3")
    sol = f2s[cell].view(-1, 40)
    assert bool((sol == sol[:, :1]).all())


@pytest.mark.parametrize("p", [1, 3])
def test_dense_blocks_match_torch_bsr(p):
    """The BSR form that ``CG(bsr_matmul=True)`` multiplies with: the DG
    matrix's dense cell blocks, column-major, as torch's own conversion gives
    them; a pattern that is not block-dense is refused."""
    from dd_solvers_b200.solvers import _dense_blocks

    s = dg.sipg(dg.uniform_mesh_2d(2), degree=p)
    A, bs = s.matrix, s.block_size
    got = _dense_blocks(A.crow_indices(), A.col_indices(), A.values(), bs)
    assert got is not None
    bptr, bcol, vals = got
    ref = A.to_sparse_bsr((bs, bs))
    assert torch.equal(bptr.to(torch.int64), ref.crow_indices())
    assert torch.equal(bcol.to(torch.int64), ref.col_indices())
    assert torch.equal(vals, ref.values().transpose(1, 2).contiguous())
    # 5-point Laplacian rows are not 2x2-block-dense
    L = sps.diags([-1, -1, 4, -1, -1], [-8, -1, 0, 1, 8], shape=(64, 64), format="csr")
    crow = torch.as_tensor(L.indptr, dtype=torch.int64)
    assert _dense_blocks(crow, torch.as_tensor(L.indices), torch.as_tensor(L.data), 2) is None


# the reference's logged higher-degree runs with S8 subdomains and coarse cells:
# degree -> (fine mesh level, cells per subdomain)
HIGHER_DEGREE_RUNS = {3: (9, 4), 5: (8, 1)}


@pytest.fixture(scope="module", params=sorted(HIGHER_DEGREE_RUNS))
def higher_degree_system(request):
    p = request.param
    m, cells = HIGHER_DEGREE_RUNS[p]
    s = dg.sipg(dg.uniform_mesh_2d(m), degree=p)
    A, b, nb = scipy_csr(s.matrix), s.load.numpy(), s.block_size
    del s
    return p, m, A, b, rs.ContiguousSchwarz(A, nb * cells, np.ones(2 * 4 ** 8, dtype=np.int64))


@pytest.mark.parametrize("kind", ["additive", "hybrid"])
def test_higher_degree_oracle_residual_history_matches_reference_log(higher_degree_system, kind):
    """The reference's P3 experiment on S9 (5,242,880 DOFs, subdomains of 40)
    and P5 experiment on S8 (2,752,512 DOFs, subdomains of 21), S8 P0 coarse
    cells, FP64: the oracle on this package's higher-degree assembly
    reproduces the first ten logged residual norms to 1e-10 (they depend on
    the GLL-warped nodes through the basis)."""
    p, m, A, b, P = higher_degree_system
    prefix = {"additive": "CG(AdditiveSchwarz(torch.float64, Inv(), CUDSS",
              "hybrid": "CG(HybridSchwarz(torch.float64, Inv(), CUDSS"}[kind]
    row = next(r for r in golden_rows() if r.get("p") == p and (r["fine"], r["solvers"], r["coarse"]) == (f"S{m}", "S8", "S8")
               and r["solver"].startswith(prefix))
    M = P.additive if kind == "additive" else P.hybrid
    T0 = P.T0 if kind == "hybrid" else None
    _, meta = rs.pcg(A, b, M=M, T0=T0, rtol=1e-9, maxiter=10, raise_on_fail=False)
    ours = np.array(meta["residual norms"])
    assert len(ours) == 10
    np.testing.assert_allclose(ours, np.array(row["residual_norms"][:10]), rtol=1e-10)


def test_logged_solver_strings_parse():
    """The reference's ``str(CG(...))`` keys of its logs map to (method,
    preconditioner precision, block precision); every converged logged
    configuration is runnable by ``dg_experiments --all``."""
    from dd_solvers_b200 import dg_experiments as de

    assert de.parse_solver("CG(HybridSchwarz(torch.float64, Inv(torch.float16), CUDSS), bsr_matmul=True)") == \
        {"method": "hybrid", "pc_precision": "f64", "precision": "f16"}
    assert de.parse_solver("CG(AdditiveSchwarz(torch.float32, Inv(), CUDSS, const_dofs_per_coarse=False), "
                           "bsr_matmul=True)") == {"method": "additive", "pc_precision": "f32", "precision": "f32"}
    with pytest.raises(ValueError):
        de.parse_solver("CG(AMGX(L1_TRUNC, None), bsr_matmul=True)")
    runs = de.logged_runs(golden_rows())
    assert {r["degree"] for r in runs} == {1, 3, 5}
    assert len({tuple(sorted(r.items())) for r in runs}) == len(runs)
    assert all(r["fine"] in ("S8", "S9", "S10", "S11") for r in runs)
    p3 = de.logged_runs(golden_rows(), degree=3)
    assert p3 and all(r["degree"] == 3 and r["fine"] == "S9" for r in p3)


def test_system_matrix_bsr_form():
    """The PCG's matrix takes the BSR form only for a block size that tiles
    the pattern densely, and keeps it in step with new values (the values of
    the differentiable solve's ``set_matrix_values``)."""
    from dd_solvers_b200.solvers import _SellMatrix, _dense_blocks

    s = dg.sipg(dg.uniform_mesh_2d(2), degree=3)
    M = _SellMatrix(s.matrix)
    assert M.use_bsr(10) and M.bsr[3] == 10 and M.bsr[2].shape == (32 + 2 * 40, 10, 10)
    assert not M.use_bsr(4) and M.bsr is None
    # block-dense at 28 x 28 (P6), but beyond the BSR kernel's block sizes: SELL stays
    assert not _SellMatrix(dg.sipg(dg.uniform_mesh_2d(1), degree=6).matrix).use_bsr(28)
    assert M.use_bsr(10)
    v = torch.randn(M.nnz, dtype=torch.float64, generator=torch.Generator().manual_seed(0))
    M.set_values(v)
    ref = _dense_blocks(M.crow32, M.col32, v, 10)
    assert torch.equal(M.bsr[2], ref[2])


def test_experiment_summary():
    from dd_solvers_b200 import dg_experiments as de

    outs = [{"iterations": 61, "reference_iterations": 61, "solve_ms_min": 40.0, "reference_a100_solve_ms_min": 160.0},
            {"iterations": 76, "reference_iterations": 75, "solve_ms_min": 50.0, "reference_a100_solve_ms_min": 250.0},
            {"iterations": 30, "solve_ms_min": 10.0}]
    assert de.summarize(outs) == {"runs": 3, "with_reference": 2, "iterations_equal": 1, "iterations_within_1": 2,
                                  "speedup_min": 4.0, "speedup_max": 5.0}


@pytest.mark.parametrize("p", [1, 2, 3, 5])
def test_sipg_consistency_with_constants(p):
    """Exact identities of the form at every degree: a constant has no
    gradient and no jumps, so A 1 vanishes on every cell away from the
    boundary (only the boundary penalty and flux act), and with f = 1 the
    load vector sums to the area of the unit square."""
    mesh = dg.uniform_mesh_2d(3)
    case = dg.TestCase("unit source", 7.0, dg._rho_continuous, lambda x, y: torch.ones_like(x))
    s = dg.sipg(mesh, case, p)
    nb = s.block_size
    r = (s.matrix @ torch.ones(s.matrix.shape[0], dtype=torch.float64)).view(mesh.n_cells, nb)
    _, (cb, _) = dg._edge_tables(mesh)
    interior = torch.ones(mesh.n_cells, dtype=torch.bool)
    interior[cb] = False
    scale = float(s.matrix.values().abs().max())
    assert float(r[interior].abs().max()) <= 1e-12 * scale
    assert float(r[~interior].abs().max()) > 1e-3 * scale  # the boundary terms are there
    assert math.isclose(float(s.load.sum()), 1.0, rel_tol=1e-13)
