"""SPD factorisation with the interface of ``dd_solvers.cudss``
(src/dd_solvers/dd_solvers/cudss.py:1-44; src/dd_solvers/cpp/cudss.cpp:34-105).

cuDSS is absent from this image. ``spd_factorize`` replaces it in two ways:

* up to ``DENSE_MAX`` rows, a dense FP64 Cholesky (cuSOLVER through
  ``torch.linalg.cholesky``) turned once into the explicit symmetric inverse,
  applied by the HBM-bound ``ddx_coarse_gemv_f64`` kernel (a tiled GEMM,
  ``ddx_coarse_gemm_f64``, for 16-64 right-hand sides);
* above that, the nested-dissection multifrontal factorisation of ``nd.py``,
  applied by ``ddx_coarse_solve_nd`` (two GEMV sweeps over the tree levels).

The batched variant factors each matrix of a block-diagonal batch the same way.
"""
from __future__ import annotations

import torch

from . import _lib as L
from . import nd

DENSE_MAX = 8192  # largest coarse size solved with a dense explicit inverse

__all__ = ["CudssSolver", "spd_factorize", "CudssBatchSolver", "spd_batch_factorize"]


def _dense_inverse(A: torch.Tensor) -> torch.Tensor:
    dense = A.to_dense().to(torch.float64) if A.layout != torch.strided else A.to(torch.float64)
    Lc, info = torch.linalg.cholesky_ex(dense)
    if int(info.max() if info.dim() else info) != 0:
        raise RuntimeError("spd_factorize: matrix is not positive definite")
    inv = torch.cholesky_inverse(Lc)
    return 0.5 * (inv + inv.transpose(-1, -2))


# K ranges the multi-RHS coarse GEMM may split its reduction into (scratch of
# GEMM_SPLIT x n x 64 doubles per solver, allocated with the factor)
GEMM_SPLIT = 16


class CudssSolver:
    def __init__(self, inverse: torch.Tensor, dtype: torch.dtype):
        self.inverse = inverse.contiguous()
        self.dtype = dtype
        self.n = inverse.shape[0]
        self.scratch = torch.empty(GEMM_SPLIT * self.n * 64, dtype=torch.float64, device=inverse.device)

    def solve_into(self, w: torch.Tensor, y: torch.Tensor, R: int, ist=None) -> None:
        """``y = A^-1 w`` for ``(n, R)`` FP64 device blocks, no allocation: a GEMV
        sweep for R < 16, the tiled GEMM (Ainv read once) for R in {16, 32, 64}."""
        if R in (16, 32, 64):
            L.call("ddx_coarse_gemm_f64", self.n, R, L.ptr(self.inverse), L.ptr(w), L.ptr(y), L.ptr(self.scratch),
                   self.scratch.numel(), L.ptr(ist), L.stream_ptr())
            return
        L.call("ddx_coarse_gemv_f64", self.n, R, L.ptr(self.inverse), L.ptr(w), L.ptr(y), L.ptr(ist),
               L.stream_ptr())

    def solve(self, rhs: torch.Tensor) -> torch.Tensor:
        L.require_cuda(rhs, "rhs")
        R = 1 if rhs.dim() == 1 else rhs.shape[1]
        w = rhs.to(torch.float64).contiguous()
        y = torch.empty_like(w)
        if R in (1, 2, 4, 8, 16, 32, 64):
            self.solve_into(w, y, R)
        else:
            for j in range(R):
                wj = w[:, j].contiguous()
                yj = torch.empty_like(wj)
                L.call("ddx_coarse_gemv_f64", self.n, 1, L.ptr(self.inverse), L.ptr(wj), L.ptr(yj), None,
                       L.stream_ptr())
                y[:, j] = yj
        return y.to(rhs.dtype)


def spd_factorize(A: torch.Tensor):
    """Factor an SPD CSR matrix on the device; the result has ``solve(rhs)``
    and ``solve_into(w, y, R, ist)``."""
    L.require_cuda(A, "A")
    if A.shape[0] <= DENSE_MAX:
        return CudssSolver(_dense_inverse(A), A.dtype)
    return nd.NDSolver(A.to(torch.float64))


class CudssBatchSolver:
    def __init__(self, solvers, sizes):
        self.solvers = solvers
        self.sizes = sizes

    def solve(self, rhs: torch.Tensor) -> torch.Tensor:
        outs, o = [], 0
        for s, n in zip(self.solvers, self.sizes):
            outs.append(s.solve(rhs[o:o + n]))
            o += n
        return torch.cat(outs)


def spd_batch_factorize(nrows, nnz, values, col_indices, row_start) -> CudssBatchSolver:
    """Block-diagonal batch given as concatenated CSR pieces (src/dd_solvers/cpp/cudss.cpp:107-247)."""
    solvers, sizes = [], []
    vo = ro = 0
    nrows_l = [int(v) for v in nrows.tolist()]
    nnz_l = [int(v) for v in nnz.tolist()]
    for n, z in zip(nrows_l, nnz_l):
        crow = row_start[ro:ro + n + 1].to(torch.int64)
        crow = crow - crow[0]
        A = torch.sparse_csr_tensor(crow, col_indices[vo:vo + z].to(torch.int64), values[vo:vo + z], size=(n, n))
        if not A.is_cuda:
            A = A.cuda()
        solvers.append(spd_factorize(A))
        sizes.append(n)
        vo += z
        ro += n + 1
    return CudssBatchSolver(solvers, sizes)
