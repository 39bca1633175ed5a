"""Setup-time CSR utilities, drop-in for ``dd_solvers.cusparse``
(src/dd_solvers/dd_solvers/cusparse.py:25-235; src/dd_solvers/cpp/cusparse.cpp:22-159).

These run once per operator and are written with torch tensor ops (device
sort/gather) instead of cuSPARSE calls.
"""
from __future__ import annotations

import torch

__all__ = ["sort_csr", "csr_to_bsr", "gather_csr"]


def sort_csr(matrix: torch.Tensor, num_parts: int | None = None) -> torch.Tensor:
    """Sorts column indices (and values) within each row; indices become int32.

    ``num_parts`` splits the work into row ranges (the reference's memory
    chunking); the result does not depend on it. The input is not modified.
    """
    rows, cols = matrix.shape
    crow = matrix.crow_indices().to(torch.int64)
    col = matrix.col_indices().to(torch.int64)
    val = matrix.values()
    if num_parts is None:
        num_parts = 1
    assert 1 <= num_parts <= max(rows, 1)
    out_col = torch.empty_like(col)
    out_val = torch.empty_like(val)
    row_of = torch.repeat_interleave(torch.arange(rows, device=crow.device), crow[1:] - crow[:-1])
    start = 0
    for part in range(num_parts):
        nr = rows // num_parts + (1 if part < rows % num_parts else 0)
        a, b = int(crow[start]), int(crow[start + nr])
        key = row_of[a:b] * cols + col[a:b]
        order = torch.argsort(key, stable=True) + a
        out_col[a:b] = col[order]
        out_val[a:b] = val[order]
        start += nr
    return torch.sparse_csr_tensor(crow.to(torch.int32), out_col.to(torch.int32), out_val, size=matrix.shape)


def gather_csr(matrix: torch.Tensor) -> torch.Tensor:
    """Sums entries with equal column within each (sorted) row
    (src/dd_solvers/dd_solvers/cusparse.py:155-235)."""
    rows, cols = matrix.shape
    crow = matrix.crow_indices()
    col = matrix.col_indices()
    val = matrix.values()
    row_of = torch.repeat_interleave(torch.arange(rows, device=crow.device),
                                     (crow[1:] - crow[:-1]).to(torch.int64))
    key = row_of * cols + col.to(torch.int64)
    ukey, counts = torch.unique_consecutive(key, return_counts=True)
    sums = torch.segment_reduce(val, "sum", lengths=counts) if val.numel() else val
    urow = ukey // cols if ukey.numel() else ukey
    ucol = ukey % cols if ukey.numel() else ukey
    new_crow = torch.zeros(rows + 1, dtype=torch.int64, device=crow.device)
    new_crow[1:] = torch.cumsum(torch.bincount(urow, minlength=rows), 0)
    return torch.sparse_csr_tensor(new_crow.to(crow.dtype), ucol.to(col.dtype), sums, size=matrix.shape)


def csr_to_bsr(matrix: torch.Tensor, block_size: int) -> torch.Tensor:
    """CSR -> BSR with column-major ``(bs, bs)`` blocks (values stride ``(bs*bs, 1, bs)``)."""
    bsr = matrix.to_sparse_bsr((block_size, block_size))
    vals = bsr.values().transpose(1, 2).contiguous().transpose(1, 2)
    return torch.sparse_bsr_tensor(bsr.crow_indices().to(torch.int32), bsr.col_indices().to(torch.int32), vals,
                                   size=matrix.shape)
