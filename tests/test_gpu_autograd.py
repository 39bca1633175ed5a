"""Differentiable solve: element-gradient kernel and adjoint gradients.

* kernel vs the NumPy formula -lambda_e^T K_e u_e (2D and 3D),
* autograd gradients vs a dense FP64 adjoint gradient at small size,
* the 512^2 Gaussian-random-field problem: directional derivatives along 16
  seeded directions in (kappa, f) vs central finite differences (h = 1e-6, FP64).
"""
import itertools

import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

from dd_solvers_b200 import partition, problems

pytestmark = pytest.mark.gpu


def _elem_grad_np(dim, n_el, u, lam):
    K = problems.q1_reference_stiffness(dim) * (1.0 / n_el) ** (dim - 2)
    m = n_el - 1
    g = np.zeros((n_el,) * dim)
    for c in itertools.product(range(n_el), repeat=dim):  # (z, y, x) / (y, x)
        cx = list(reversed(c))  # x, y, z
        ul, ll = np.zeros(2 ** dim), np.zeros(2 ** dim)
        for a in range(2 ** dim):
            p = [cx[d] + ((a >> d) & 1) for d in range(dim)]
            if all(1 <= q <= m for q in p):
                idx = 0
                for d in reversed(range(dim)):
                    idx = idx * m + p[d] - 1
                ul[a], ll[a] = u[idx], lam[idx]
        g[c] = -ll @ K @ ul
    return g


@pytest.mark.parametrize("dim,n_el", [(2, 9), (3, 5)])
def test_elem_grad_kernel(cuda, dim, n_el):
    from dd_solvers_b200 import Q1Diffusion

    op = Q1Diffusion(dim, n_el, cuda)
    rng = np.random.default_rng(dim)
    u, lam = rng.standard_normal(op.n), rng.standard_normal(op.n)
    g = op.elem_grad(torch.as_tensor(u, device=cuda), torch.as_tensor(lam, device=cuda)).cpu().numpy()
    assert np.allclose(g, _elem_grad_np(dim, n_el, u, lam), rtol=1e-13, atol=1e-13)


def _setup(cuda, n_el, parts, kappa):
    import dd_solvers_b200 as dd

    op = dd.Q1Diffusion(2, n_el, cuda)
    A = problems.q1_grid(2, n_el, kappa).matrix
    P = problems.q1_grid(2, n_el)
    owner, nparts = partition.box_owner(P.interior_shape, parts)
    sub_ptr, sub_idx = partition.overlapping_subdomains(A, owner, nparts, 1)
    # The preconditioner is built once and reused for other kappa: it must stay
    # SPD for any A, which the additive form is (the hybrid projection is not).
    cg = dd.CG(dd.AdditiveSchwarz(torch.float64, dd.Inv(), dd.CUDSS()), rtol=1e-12, maxiter=5000)
    cg.setup(op.matrix(torch.as_tensor(kappa, device=cuda)), subdomains=(sub_ptr, sub_idx), owner=owner,
             block_size=1)
    return op, cg, A


def test_gradient_matches_dense_adjoint(cuda):
    import dd_solvers_b200 as dd

    n_el = 24
    rng = np.random.default_rng(0)
    kappa = np.exp(0.5 * rng.standard_normal((n_el, n_el)))
    f = rng.uniform(-1, 1, (n_el - 1) ** 2)
    ut = rng.standard_normal((n_el - 1) ** 2) * 1e-3
    op, cg, A = _setup(cuda, n_el, 4, kappa)
    k_t = torch.tensor(kappa, device=cuda, requires_grad=True)
    f_t = torch.tensor(f, device=cuda, requires_grad=True)
    u = dd.DiffusionSolve.apply(k_t, f_t, op, cg)
    loss = ((u - torch.as_tensor(ut, device=cuda)) ** 2).sum()
    loss.backward()
    # dense FP64 adjoint
    h = 1.0 / n_el
    w = np.full(A.shape[0], h * h)
    Ad = A.toarray()
    ud = np.linalg.solve(Ad, w * f)
    lam = np.linalg.solve(Ad, 2 * (ud - ut))
    gk = _elem_grad_np(2, n_el, ud, lam)
    gf = w * lam
    assert np.allclose(u.detach().cpu().numpy(), ud, rtol=1e-9, atol=1e-14)
    assert np.linalg.norm(k_t.grad.cpu().numpy() - gk) <= 1e-8 * np.linalg.norm(gk)
    assert np.linalg.norm(f_t.grad.cpu().numpy() - gf) <= 1e-8 * np.linalg.norm(gf)


def test_grf_gradient_central_differences(cuda):
    """512^2 cells, kappa = exp(g) with g a squared-exponential GRF (l = 0.1),
    f = 1, loss ||u - u_t||^2 with u_t from a second field; 16 directions."""
    import dd_solvers_b200 as dd

    n_el = 512
    g = problems.gaussian_random_field(n_el, 0.1, seed=0)
    gt = problems.gaussian_random_field(n_el, 0.1, seed=1)
    kappa, kappa_t = np.exp(g), np.exp(gt)
    op, cg, _ = _setup(cuda, n_el, 16, kappa)
    f = torch.ones(op.n, dtype=torch.float64, device=cuda)
    with torch.no_grad():
        ut = dd.DiffusionSolve.apply(torch.as_tensor(kappa_t, device=cuda), f, op, cg)
    k0 = torch.as_tensor(kappa, device=cuda)

    def loss_of(k, ff):
        u = dd.DiffusionSolve.apply(k, ff, op, cg)
        return ((u - ut) ** 2).sum()

    k_t = k0.clone().requires_grad_(True)
    f_t = f.clone().requires_grad_(True)
    L0 = loss_of(k_t, f_t)
    L0.backward()
    gk, gf = k_t.grad, f_t.grad
    rng = np.random.default_rng(123)
    h = 1e-6
    worst = 0.0
    for _ in range(16):
        dk = torch.as_tensor(rng.standard_normal(kappa.shape), device=cuda) * k0  # relative perturbation
        df = torch.as_tensor(rng.standard_normal(op.n), device=cuda)
        with torch.no_grad():
            lp = float(loss_of(k0 + h * dk, f + h * df))
            lm = float(loss_of(k0 - h * dk, f - h * df))
        fd = (lp - lm) / (2 * h)
        ad = float((gk * dk).sum() + (gf * df).sum())
        worst = max(worst, abs(fd - ad) / max(abs(ad), 1e-30))
    # Error budget: each of the two solves per difference stops at rtol 1e-12,
    # leaving ~1e-11 relative error in L, amplified by 1/(2h) = 5e5 -> ~1e-5.
    assert worst <= 1e-4, worst
