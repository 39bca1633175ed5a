"""Differentiable Schwarz-PCG solve of a Q1 diffusion problem.

``DiffusionSolve.apply(kappa, f, op, cg)`` returns ``u = A(kappa)^{-1} (w * f)``
where ``A(kappa) = sum_e kappa_e K_e`` is the Q1 stiffness on a uniform grid
(Dirichlet nodes eliminated) and ``w`` the lumped nodal mass. The backward
pass solves the adjoint system with the same preconditioned CG (A is
symmetric): ``A lambda = dL/du``, then

* ``dL/df = w * lambda``
* ``dL/dkappa_e = -lambda_e^T K_e u_e`` by the ``ddx_elem_grad_q1`` kernel.

The reference has no differentiable solve; this follows the standard adjoint
method. The preconditioner is built once (for a representative kappa) and
reused: PCG converges to ``A(kappa)^{-1} b`` for any SPD preconditioner, so
only the matrix values are refreshed per call (``CG.set_matrix_values``).
Use ``AdditiveSchwarz`` for a reused preconditioner: it is SPD whatever the
current matrix, whereas ``HybridSchwarz`` projects with ``R0 A`` of the matrix
it was built for and must be rebuilt when kappa changes.
"""
from __future__ import annotations

import itertools

import numpy as np
import torch

from . import _lib as L
from . import problems


class Q1Diffusion:
    """Q1 stiffness with per-element coefficient, assembled on the device.

    The CSR pattern (9-point 2D / 27-point 3D stencil, x-fastest interior
    numbering) is fixed; ``assemble(kappa)`` returns the values in CSR order.
    """

    def __init__(self, dim: int, n_el: int, device):
        self.dim, self.n_el, self.device = dim, n_el, torch.device(device)
        self.m = n_el - 1
        self.n = self.m ** dim
        P = problems.q1_grid(dim, n_el)
        A = P.matrix
        self.crow = torch.as_tensor(A.indptr.astype(np.int64), device=self.device)
        self.col = torch.as_tensor(A.indices.astype(np.int64), device=self.device)
        self.h = 1.0 / n_el
        kref = problems.q1_reference_stiffness(dim)
        self.kref = torch.as_tensor(kref, device=self.device).contiguous()
        self.mass = torch.full((self.n,), self.h ** dim, dtype=torch.float64, device=self.device)
        # stencil terms: (offset id, cell slice per axis, coefficient)
        Kh = kref * self.h ** (dim - 2)
        offsets = list(itertools.product((-1, 0, 1), repeat=dim))
        self.terms = []
        for oi, off in enumerate(offsets):
            choices = [[s for s in (0, 1) if s - o in (0, 1)] for o in off]
            for shifts in itertools.product(*choices):
                la = lb = 0
                for d in range(dim):
                    bit = dim - 1 - d
                    la |= (1 - shifts[d]) << bit
                    lb |= (1 - shifts[d] + off[d]) << bit
                self.terms.append((oi, tuple(shifts), float(Kh[la, lb])))
        # gather index from the dense (noff, n) stencil table to CSR order
        m = self.m
        grids = np.meshgrid(*[np.arange(m)] * dim, indexing="ij")
        valid = np.empty((len(offsets), self.n), dtype=bool)
        for oi, off in enumerate(offsets):
            ok = np.ones((m,) * dim, dtype=bool)
            for d in range(dim):
                q = grids[d] + off[d]
                ok &= (q >= 0) & (q < m)
            valid[oi] = ok.ravel()
        flat = (np.arange(len(offsets))[:, None] * self.n + np.arange(self.n)[None, :]).T[valid.T]
        self.gather = torch.as_tensor(flat, device=self.device)
        self.noff = len(offsets)

    def assemble(self, kappa: torch.Tensor) -> torch.Tensor:
        """CSR values of A(kappa); kappa has shape (n_el,)*dim (x fastest)."""
        kappa = kappa.to(self.device, torch.float64)
        m = self.m
        vals = torch.zeros((self.noff,) + (m,) * self.dim, dtype=torch.float64, device=self.device)
        for oi, shifts, coef in self.terms:
            sl = tuple(slice(s, s + m) for s in shifts)
            vals[oi] += coef * kappa[sl]
        return vals.reshape(-1)[self.gather]

    def matrix(self, kappa: torch.Tensor) -> torch.Tensor:
        return torch.sparse_csr_tensor(self.crow, self.col, self.assemble(kappa), (self.n, self.n))

    def elem_grad(self, u: torch.Tensor, lam: torch.Tensor) -> torch.Tensor:
        """-lambda_e^T K_e u_e per cell, shape (n_el,)*dim."""
        L.require_cuda(u, "u")
        g = torch.empty((self.n_el,) * self.dim, dtype=torch.float64, device=self.device)
        u = u.to(torch.float64).contiguous()
        lam = lam.to(torch.float64).contiguous()
        L.call("ddx_elem_grad_q1", self.dim, self.n_el, L.ptr(u), L.ptr(lam), L.ptr(self.kref), L.ptr(g),
               L.stream_ptr())
        return g


class DiffusionSolve(torch.autograd.Function):
    """u = A(kappa)^{-1} (mass * f); gradients by the adjoint PCG solve."""

    @staticmethod
    def forward(ctx, kappa, f, op: Q1Diffusion, cg):
        vals = op.assemble(kappa)
        cg.set_matrix_values(vals)
        b = (op.mass * f.to(torch.float64)).contiguous()
        u, _ = cg.solve(b)
        ctx.op, ctx.cg = op, cg
        ctx.save_for_backward(u, vals)
        ctx.kappa_dtype, ctx.f_dtype = kappa.dtype, f.dtype
        return u

    @staticmethod
    def backward(ctx, gu):
        u, vals = ctx.saved_tensors
        op, cg = ctx.op, ctx.cg
        cg.set_matrix_values(vals)
        lam, _ = cg.solve(gu.to(torch.float64).contiguous())
        grad_f = (op.mass * lam).to(ctx.f_dtype) if ctx.needs_input_grad[1] else None
        grad_k = op.elem_grad(u, lam).to(ctx.kappa_dtype) if ctx.needs_input_grad[0] else None
        return grad_k, grad_f, None, None
