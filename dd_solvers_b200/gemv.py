"""Batched GEMV custom op, drop-in for ``dd_solvers.gemv`` (src/dd_solvers/dd_solvers/gemv.py:4-30).

``gemv_strided_batched(matrices, vectors, use_shared_memory=None)`` computes
``out[b] = M_b v_b`` for column-major ``(N, k, k)`` matrices in FP16/BF16/FP32/FP64
and ``(N, k)`` vectors in FP32/FP64, converting matrix entries to the vector
type and accumulating in it. ``use_shared_memory`` is accepted for
compatibility; the sm_100a kernel always stages the vectors in shared memory.
"""
from __future__ import annotations

import torch

from . import _lib as L


@torch.library.custom_op("dd_solvers_b200::gemv_strided_batched", mutates_args=())
def gemv_strided_batched(matrices: torch.Tensor, vectors: torch.Tensor,
                         use_shared_memory: bool | None = None) -> torch.Tensor:
    if vectors.dtype not in (torch.float32, torch.float64):
        raise ValueError("Unsupported data type")
    if not (matrices.dim() == 3 and vectors.dim() == 2 and matrices.size(0) == vectors.size(0)
            and matrices.size(1) == matrices.size(2) and matrices.size(1) == vectors.size(1)):
        raise RuntimeError("Input tensors must have compatible dimensions: (n, k, k) and (n, k)")
    k = matrices.size(1)
    if not (matrices.stride(1) == 1 and (matrices.stride(2) == k or k <= 1)):
        raise RuntimeError("Matrices must be in column-major format")
    L.require_cuda(matrices, "matrices")
    L.require_cuda(vectors, "vectors")
    vec = vectors.contiguous()
    out = torch.empty_like(vec)
    L.call("ddx_gemv_strided_batched", matrices.size(0), k, L.ptr(matrices), L.DTYPE_CODE[matrices.dtype],
           L.ptr(vec), L.ptr(out), L.DTYPE_CODE[vec.dtype], L.stream_ptr())
    return out


@gemv_strided_batched.register_fake
def _gemv_strided_batched_fake(matrices: torch.Tensor, vectors: torch.Tensor,
                               use_shared_memory: bool | None = None) -> torch.Tensor:
    if matrices.ndim != 3 or vectors.ndim != 2:
        raise RuntimeError("matrices must be 3D and vectors must be 2D")
    if matrices.shape[0] != vectors.shape[0]:
        raise RuntimeError("matrices and vectors must have the same batch size")
    return torch.empty_like(vectors)
