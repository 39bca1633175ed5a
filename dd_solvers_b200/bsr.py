"""Block-sparse (BSR) matrix-vector product, drop-in for ``FastBSR``
(src/dd_solvers/dd_solvers/bsr.py:15-25, 237-244).

The reference registers several numba kernels; here every backend name maps to
the sm_100a ``ddx_spmv_bsr`` kernel: one scalar row per lane, floor(32 / bs)
block rows per warp, so the bs lanes of a block row read each column of the
column-major blocks as consecutive values and x is a broadcast; no cross-lane
reduction. ``CG(bsr_matmul=True)`` with a block size >= 2 runs its products
through the same kernel.
"""
from __future__ import annotations

import torch

from . import _lib as L

__all__ = ["FastBSR"]


class FastBSR:
    matmul_backends = {"warp_per_block_row": None, "row_per_thread_irrespective": None}

    def __init__(self, matrix: torch.Tensor, backend: str = "row_per_thread_irrespective"):
        assert matrix.is_cuda
        assert matrix.layout is torch.sparse_bsr
        if backend not in self.matmul_backends:
            raise KeyError(backend)
        vals = matrix.values()
        self.bs = vals.shape[1]
        assert vals.shape[1] == vals.shape[2]
        # column-major blocks: element (r, c) of block b at b*bs*bs + c*bs + r
        self.vals = vals.transpose(1, 2).contiguous()
        self.crow = matrix.crow_indices().to(torch.int32)
        self.col = matrix.col_indices().to(torch.int32)
        self.shape = matrix.shape
        self.dtype = vals.dtype

    def __matmul__(self, x: torch.Tensor) -> torch.Tensor:
        xx = x.to(self.dtype).contiguous()
        y = torch.empty(self.shape[0], dtype=self.dtype, device=x.device)
        L.call("ddx_spmv_bsr", self.crow.numel() - 1, self.bs, L.ptr(self.crow), L.ptr(self.col), L.ptr(self.vals),
               L.ptr(xx), L.ptr(y), L.DTYPE_CODE[self.dtype], L.stream_ptr())
        return y
