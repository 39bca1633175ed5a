"""GPU tests of the nested-dissection coarse solver and of the reference's DG
experiments run end to end (assembly, ordering, setup, PCG) on the device."""
import json
import os
import sys

import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from dd_solvers_b200 import cudss, dg_experiments, nd  # noqa: E402
from nd_emulation import emulate_solve  # noqa: E402
from test_nd import CASES, lap2d  # noqa: E402

pytestmark = pytest.mark.gpu


def to_dev(A):
    A = A.tocsr()
    A.sort_indices()
    return torch.sparse_csr_tensor(torch.as_tensor(A.indptr, dtype=torch.int64),
                                   torch.as_tensor(A.indices, dtype=torch.int64),
                                   torch.as_tensor(A.data, dtype=torch.float64), A.shape).cuda()


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("R", [1, 3, 16])
@pytest.mark.parametrize("tree", ["merged", "full"])
def test_nd_solve_matches_sparse_lu(case, R, tree):
    """One merged front (the default for these small cases), or the full
    separator tree cut into 8-row items, whose upper levels take the gather
    launch."""
    A = CASES[case]()
    solver = nd.NDSolver(to_dev(A), leaf=32 if tree == "merged" else 16, top_merge=None if tree == "merged" else 0)
    if tree == "full":
        solver.set_items(512, 8)
        assert solver.sym.gat_level_ptr[-1] > 0
    w = np.random.default_rng(R).standard_normal((A.shape[0], R))
    x = solver.solve(torch.as_tensor(w, device="cuda")).cpu().numpy()
    ref = spla.splu(A.tocsc()).solve(w)
    assert np.abs(x - ref).max() <= 1e-12 * np.abs(ref).max()


def test_nd_sweep_variants_agree_bitwise(monkeypatch):
    """Operator rows staged in shared memory or read from global memory, f
    gathered by the gather launch or inside the forward items, early or late
    release of the next level: the same sums in the same order, so the same
    bits."""
    A = lap2d(45)
    solver = nd.NDSolver(to_dev(A), leaf=16, top_merge=0)
    solver.set_items(512, 8)
    assert solver.gather and solver.plan.release_early == 1 and (solver.fwd_level_gmax >= 0).any()
    w = torch.randn(A.shape[0], 3, dtype=torch.float64, device="cuda")
    ref = solver.solve(w)
    for knob in ("STAGE", "GATHER", "RELEASE"):
        monkeypatch.setattr(nd, knob, False)
        solver.set_items(512, 8)
        assert torch.equal(solver.solve(w), ref), knob
    assert not solver.gather and solver.plan.release_early == 0 and (solver.fwd_level_gmax < 0).all()


def test_nd_solve_matches_host_emulation_and_is_deterministic():
    A = lap2d(60)
    At = to_dev(A)
    solver = nd.NDSolver(At, leaf=64)
    w = torch.randn(A.shape[0], 4, dtype=torch.float64, device="cuda")
    x1 = solver.solve(w)
    x2 = solver.solve(w)
    assert torch.equal(x1, x2)
    xe = emulate_solve(solver.sym, solver.G.cpu().numpy(), solver.GT.cpu().numpy(), w.cpu().numpy())
    np.testing.assert_allclose(x1.cpu().numpy(), xe, rtol=1e-12, atol=1e-12 * np.abs(xe).max())


def test_large_coarse_matrix_takes_the_sparse_path():
    A = lap2d(100)  # 10,000 rows > DENSE_MAX
    assert A.shape[0] > cudss.DENSE_MAX
    s = cudss.spd_factorize(to_dev(A))
    assert isinstance(s, nd.NDSolver)
    w = torch.randn(A.shape[0], dtype=torch.float64, device="cuda")
    x = s.solve(w).cpu().numpy()
    ref = spla.splu(A.tocsc()).solve(w.cpu().numpy())
    assert np.abs(x - ref).max() <= 1e-12 * np.abs(ref).max()


LOG = os.path.join(ROOT, "tests", "golden", "dg_experiments.json")


@pytest.mark.parametrize("method", ["additive", "hybrid"])
def test_dg_experiment_reproduces_reference_log(method):
    """Fine S10 (6.29M DOFs), 131,072 subdomains of 48 DOFs and a 131,072-DOF
    P0 coarse space, FP64: the GPU run reproduces the reference's logged
    iteration count and residual history."""
    log = json.load(open(LOG))
    out = dg_experiments.run("S10", "S8", "S8", method, "f64", reps=1, log=log)
    assert out["dofs"] == 6291456 and out["nnz"] == 75460608
    assert abs(out["iterations"] - out["reference_iterations"]) <= 1
    assert out["history_max_rel_diff_first10"] < 1e-10
    # later norms drift only by rounding (hybrid converges to ~1e-10 of r0)
    assert out["history_max_rel_diff"] < 1e-2


@pytest.mark.parametrize("precision,expected", [("f16", 61), ("bf16", 62), ("f32", 61)])
def test_dg_experiment_mixed_precision_iterations(precision, expected):
    """Low-precision blocks (FP64 preconditioner, plain CG as the reference
    runs it): the reference's logged iteration counts for S10 / S8 / S8."""
    log = json.load(open(LOG))
    out = dg_experiments.run("S10", "S8", "S8", "hybrid", precision, reps=1, log=log)
    assert out["reference_iterations"] == expected
    assert abs(out["iterations"] - expected) <= 1
    assert out["history_max_rel_diff_first10"] < 1e-5


@pytest.mark.parametrize("p,fine,cells,method", [(3, "S9", "S8", "hybrid"), (3, "S9", "S8", "additive"),
                                                  (5, "S8", "S7", "hybrid"), (5, "S8", "S7", "additive")])
def test_dg_higher_degree_experiment_reproduces_reference_log(p, fine, cells, method):
    """The reference's P3 (S9, 5.24M DOFs, 10 per cell) and P5 (S8, 2.75M
    DOFs, 21 per cell) experiments, FP64: its logged size, iteration count and
    residual history (GLL-warped nodes, exact quadrature)."""
    log = json.load(open(LOG))
    out = dg_experiments.run(fine, cells, cells, method, "f64", reps=1, log=log, degree=p)
    size = {3: (5242880, 209510400), 5: (2752512, 230759424)}[p]
    assert (out["dofs"], out["nnz"]) == size
    assert abs(out["iterations"] - out["reference_iterations"]) <= 1
    assert out["history_max_rel_diff_first10"] < 1e-10
    # later norms drift only by rounding (the reference ran BSR products on an A100)
    assert out["history_max_rel_diff"] < 1e-2


@pytest.mark.parametrize("p,fine,precision,expected", [(3, "S9", "f16", 131), (5, "S8", "bf16", 152)])
def test_dg_higher_degree_mixed_precision_iterations(p, fine, precision, expected):
    """Low-precision blocks on the P3 / P5 problems with S8 subdomains and
    coarse cells: the reference's logged iteration counts."""
    log = json.load(open(LOG))
    out = dg_experiments.run(fine, "S8", "S8", "hybrid", precision, reps=1, log=log, degree=p)
    assert out["reference_iterations"] == expected
    assert abs(out["iterations"] - expected) <= 1
    assert out["history_max_rel_diff_first10"] < 1e-6


@pytest.mark.parametrize("p,fine", [(1, "S6"), (3, "S5"), (5, "S4")])
def test_cg_bsr_products_match_csr(p, fine):
    """``CG(bsr_matmul=True)`` on a DG matrix multiplies in BSR form (the cell
    blocks, ``ddx_spmv_bsr``) with the PCG epilogue as a separate pass; the
    same solve with ``bsr_matmul=False`` (CSR products with fused epilogues)
    takes the same iterations and reaches the same solution. Residual
    replacement exercises the r = b - A x epilogue."""
    import dd_solvers_b200 as dd

    A, b, kw = dg_experiments.build(fine, "S3", "S3", degree=p)
    nb = (p + 1) * (p + 2) // 2
    runs = {}
    for name, opts in {"bsr": {}, "csr": {"bsr_matmul": False}, "bsr_replace": {"replace_every": 7}}.items():
        cg = dd.CG(dd.HybridSchwarz(torch.float64, dd.Inv(), dd.CUDSS()), rtol=1e-10, **opts)
        cg.setup(A, **kw)
        assert (cg.matrix.bsr is not None) == (name != "csr")
        x, meta = cg.solve(b)
        runs[name] = (x, meta)
        if name == "bsr":
            v = torch.randn(A.shape[0], dtype=torch.float64, device="cuda")
            ref = (A @ v[:, None])[:, 0]
            got = cg.matrix @ v
            assert float((got - ref).abs().max()) <= 1e-12 * float(ref.abs().max())
            assert cg.matrix.bsr[3] == nb
        cg.destroy()
    xb, mb = runs["bsr"]
    xc, mc = runs["csr"]
    assert mb["iterations"] == mc["iterations"]
    assert float(torch.linalg.norm(xb - xc)) <= 1e-9 * float(torch.linalg.norm(xc))
    hb, hc = np.array(mb["residual norms"][:10]), np.array(mc["residual norms"][:10])
    np.testing.assert_allclose(hb, hc, rtol=1e-11)
    xr, mr = runs["bsr_replace"]
    assert abs(mr["iterations"] - mc["iterations"]) <= 1
    assert float(torch.linalg.norm(xr - xc)) <= 1e-8 * float(torch.linalg.norm(xc))


def test_dg_experiment_quadrilateral_cells():
    """Solver and coarse cells on the C-level quadrilateral grids (the DOFs are
    permuted into (coarse, solver) groups first): S9 fine, C8 solvers (24 DOFs
    each), C6 coarse cells; the PCG converges and the grouping is consistent."""
    A, b, kw = dg_experiments.build("S9", "C8", "C6")
    assert kw["dofs_per_solver"] == 24
    assert int(kw["solvers_per_coarse"].sum()) == 4 ** 8
    assert bool((kw["solvers_per_coarse"] == 16).all())
    out = dg_experiments.run("S9", "C8", "C6", "hybrid", "f64", reps=1)
    assert out["iterations"] < 200


def test_reference_experiment_factory_case():
    """``src/experiments/tests/test_experiments.py:10-41``: fine S3, the direct
    coarse-solver interface on the whole system, and CG(AdditiveSchwarz(float32,
    Inv(float16), CUDSS)) with C3 subdomains and one C0 coarse cell; both reach
    a residual below 1e-6 and an L2 error below 0.5."""
    import dd_solvers_b200 as dd
    from dd_solvers_b200 import dg

    A, b, kw, perm = dg_experiments.build("S3", "C3", "C0", return_perm=True)
    inv = torch.empty_like(perm)
    inv[perm] = torch.arange(perm.numel(), device=perm.device)
    mesh = dg.uniform_mesh_2d(3)
    case = dg.CONTINUOUS_COEFFICIENT_2D

    direct = dd.CUDSS()
    direct.setup(A)
    x_direct, _ = direct.solve(b)
    cg = dd.CG(dd.AdditiveSchwarz(torch.float32, dd.Inv(torch.float16), dd.CUDSS()))
    cg.setup(A, **kw)
    x_cg, meta = cg.solve(b)
    for x in (x_direct, x_cg):
        res = float(torch.linalg.norm(torch.sparse.mm(A, x[:, None])[:, 0] - b))
        assert res < 1e-6, res
        err = dg.l2_error(mesh, x[inv].cpu(), case.solution)
        assert err < 0.5, err
