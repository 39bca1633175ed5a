"""Subdomain decompositions and coarse spaces (host-side setup).

The reference groups DOFs into equal, contiguous, non-overlapping blocks after a
permutation (``asm_permutation``, ``src/dd_solvers/dd_solvers/solvers.py:541-551``)
and uses a piecewise-constant (P0) coarse space whose restriction sums each group
of consecutive blocks (``solvers.py:817-825``). The workloads measured here need
overlap, uneven subdomains and a Q1 coarse space, so subdomains are described by
explicit index sets instead:

* a subdomain set is ``(sub_ptr, sub_idx)``: subdomain ``i`` holds the global
  DOFs ``sub_idx[sub_ptr[i]:sub_ptr[i+1]]`` in ascending order (CSR-like);
* ``owner[j]`` is the non-overlapping part that DOF ``j`` belongs to; overlap
  is added as layers of matrix-graph neighbours;
* a coarse space is a restriction ``R0`` (``n_c x n`` CSR); the P0 space of the
  reference is ``R0[c, j] = 1`` iff DOF ``j`` is owned by a part in coarse group
  ``c``.

With zero overlap and owners equal to contiguous equal blocks these reduce to
the reference's layout exactly.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sps


def box_owner(interior_shape: tuple, parts_per_axis: int | tuple) -> tuple[np.ndarray, int]:
    """Node partition of a structured interior grid into boxes.

    ``interior_shape`` is ``(m,)*dim`` (x fastest in the DOF numbering). With
    ``P`` parts per axis, interior node ``p`` (1-based grid index) goes to part
    ``min(p // (n_el / P), P - 1)``, i.e. the element-box containing the node's
    lower-left cell, so interior subdomains own ``(n_el/P)**dim`` nodes.
    Returns ``(owner, n_parts)``; part ids are lexicographic with x fastest.
    """
    dim = len(interior_shape)
    if np.isscalar(parts_per_axis):
        parts_per_axis = (int(parts_per_axis),) * dim
    owner = np.zeros(interior_shape, dtype=np.int64)
    stride = 1
    # interior_shape axes are (.., y, x): axis dim-1 is x
    for d in range(dim - 1, -1, -1):
        m = interior_shape[d]
        P = parts_per_axis[d]
        n_el = m + 1
        width = n_el / P
        p = np.arange(1, m + 1)
        part = np.minimum((p // width).astype(np.int64), P - 1)
        shape = [1] * dim
        shape[d] = m
        owner = owner + part.reshape(shape) * stride
        stride *= P
    return owner.ravel().astype(np.int32), int(np.prod(parts_per_axis))


def rcb_owner(coords: np.ndarray, n_parts: int) -> np.ndarray:
    """Recursive coordinate bisection at the bounding-box midpoint.

    Each part is split along the longest side of its bounding box at the
    geometric midpoint (not the median), so node jitter makes the part sizes
    uneven. ``n_parts`` must be a power of two. Returns ``owner`` (n,) int32
    with parts numbered by their bisection path.
    """
    assert n_parts & (n_parts - 1) == 0, "n_parts must be a power of two"
    n = coords.shape[0]
    owner = np.zeros(n, dtype=np.int64)
    levels = int(np.log2(n_parts))
    for _ in range(levels):
        order = np.argsort(owner, kind="stable")
        o_sorted = owner[order]
        starts = np.flatnonzero(np.r_[True, o_sorted[1:] != o_sorted[:-1]])
        c_sorted = coords[order]
        lo = np.minimum.reduceat(c_sorted, starts, axis=0)
        hi = np.maximum.reduceat(c_sorted, starts, axis=0)
        axis = np.argmax(hi - lo, axis=1)
        mid = 0.5 * (lo + hi)[np.arange(len(starts)), axis]
        counts = np.diff(np.r_[starts, n])
        ax_pt = np.repeat(axis, counts)
        mid_pt = np.repeat(mid, counts)
        side = (c_sorted[np.arange(n), ax_pt] >= mid_pt).astype(np.int64)
        new = np.empty(n, dtype=np.int64)
        new[order] = o_sorted * 2 + side
        owner = new
    return owner.astype(np.int32)


def overlapping_subdomains(A: sps.csr_matrix, owner: np.ndarray, n_parts: int,
                           overlap: int) -> tuple[np.ndarray, np.ndarray]:
    """Grow each owned set by ``overlap`` layers of matrix-graph neighbours.

    Returns ``(sub_ptr int64 (n_parts+1,), sub_idx int32)`` with each subdomain's
    DOFs sorted ascending.
    """
    n = A.shape[0]
    S = sps.csr_matrix((np.ones(n, dtype=np.int8), (owner.astype(np.int64), np.arange(n))),
                       shape=(n_parts, n))
    if overlap > 0:
        G = A.copy()
        G.data = np.ones_like(G.data, dtype=np.int8)
        G = G.astype(np.int8)
        for _ in range(overlap):
            S = (S @ G).astype(bool).astype(np.int8)
    S = S.tocsr()
    S.sort_indices()
    return S.indptr.astype(np.int64), S.indices.astype(np.int32)


def contiguous_subdomains(n: int, dofs_per_solver: int) -> tuple[np.ndarray, np.ndarray]:
    """Equal contiguous blocks: the reference's implicit layout (``solvers.py:814``)."""
    assert n % dofs_per_solver == 0
    N = n // dofs_per_solver
    return (np.arange(N + 1, dtype=np.int64) * dofs_per_solver, np.arange(n, dtype=np.int32))


def p0_restriction(owner: np.ndarray, n_parts: int, parts_to_coarse: np.ndarray | None = None) -> sps.csr_matrix:
    """P0 coarse restriction: ``R0[c, j] = 1`` iff ``owner[j]`` belongs to coarse group ``c``.

    ``parts_to_coarse`` maps parts to coarse groups (default: identity), the
    counterpart of the reference's ``solvers_to_coarse`` (``solvers.py:722-724``).
    """
    n = owner.shape[0]
    grp = owner if parts_to_coarse is None else np.asarray(parts_to_coarse)[owner]
    n_c = n_parts if parts_to_coarse is None else int(np.max(parts_to_coarse)) + 1
    R = sps.csr_matrix((np.ones(n), (grp.astype(np.int64), np.arange(n))), shape=(n_c, n))
    R.sort_indices()
    return R


def q1_coarse_restriction(dim: int, n_el: int, parts_per_axis: int) -> sps.csr_matrix:
    """Restriction ``R0 = P^T`` for a Q1 coarse grid on the subdomain vertices.

    Coarse nodes sit at multiples of ``H = n_el / parts_per_axis`` cells; the
    coarse boundary nodes are Dirichlet and dropped, leaving
    ``(parts_per_axis - 1)**dim`` coarse DOFs. ``P`` interpolates coarse nodal
    values multilinearly to the fine interior nodes.
    """
    P_ax = parts_per_axis
    assert n_el % P_ax == 0
    H = n_el // P_ax
    m = n_el - 1
    mc = P_ax - 1
    # 1D interpolation matrix (m x mc): fine node p (1..m), coarse node c (1..mc)
    rows, cols, vals = [], [], []
    for p in range(1, m + 1):
        c0 = p // H
        t = (p - c0 * H) / H
        for c, w in ((c0, 1.0 - t), (c0 + 1, t)):
            if 1 <= c <= mc and w != 0.0:
                rows.append(p - 1)
                cols.append(c - 1)
                vals.append(w)
    P1 = sps.csr_matrix((vals, (rows, cols)), shape=(m, mc))
    P = P1
    for _ in range(dim - 1):
        P = sps.kron(P, P1, format="csr")  # later axes are slower; x fastest
    R = P.T.tocsr()
    R.sort_indices()
    return R


# ---------------------------------------------------------------------------
# the same decompositions on the device (torch; any device)
# ---------------------------------------------------------------------------

def rcb_owner_device(coords, n_parts: int):
    """``rcb_owner`` on a torch ``(n, dim)`` FP64 tensor: per level, the parts'
    bounding boxes by segmented min/max, the longest axis (first on ties, as
    ``np.argmax``), the midpoint, and the side of every node. The arithmetic is
    the same, so the owners are identical to ``rcb_owner``."""
    import torch

    assert n_parts & (n_parts - 1) == 0, "n_parts must be a power of two"
    n, dim = coords.shape
    dev = coords.device
    owner = torch.zeros(n, dtype=torch.int64, device=dev)
    ar = torch.arange(n, device=dev)
    for lv in range(int(np.log2(n_parts))):
        P = 1 << lv
        idx = owner[:, None].expand(n, dim)
        lo = torch.full((P, dim), float("inf"), dtype=coords.dtype, device=dev).scatter_reduce(
            0, idx, coords, "amin", include_self=True)
        hi = torch.full((P, dim), float("-inf"), dtype=coords.dtype, device=dev).scatter_reduce(
            0, idx, coords, "amax", include_self=True)
        axis = torch.argmax(hi - lo, dim=1)
        mid = 0.5 * (lo + hi)[torch.arange(P, device=dev), axis]
        side = (coords[ar, axis[owner]] >= mid[owner]).to(torch.int64)
        owner = owner * 2 + side
    return owner.to(torch.int32)


def overlapping_subdomains_device(crow, col, owner, n_parts: int, overlap: int):
    """``overlapping_subdomains`` from a device CSR pattern (``crow``, ``col``) and
    owners: the part-by-DOF incidence grown by ``overlap`` sparse products with
    the matrix graph (cuSPARSE SpGEMM through torch), columns sorted. Returns
    ``(sub_ptr int64, sub_idx int32)`` torch tensors on the same device."""
    import torch

    from .setup_ops import spgemm_sorted

    dev = crow.device
    n = crow.numel() - 1
    order = torch.argsort(owner.to(torch.int64), stable=True)
    counts = torch.bincount(owner.to(torch.int64), minlength=n_parts)
    ptr = torch.zeros(n_parts + 1, dtype=torch.int64, device=dev)
    ptr[1:] = torch.cumsum(counts, 0)
    S = torch.sparse_csr_tensor(ptr, order, torch.ones(n, dtype=torch.float64, device=dev), (n_parts, n))
    G = torch.sparse_csr_tensor(crow.to(torch.int64), col.to(torch.int64),
                                torch.ones(col.numel(), dtype=torch.float64, device=dev), (n, n))
    for _ in range(overlap):
        p, c, _v = spgemm_sorted(S, G)
        S = torch.sparse_csr_tensor(p, c, torch.ones(c.numel(), dtype=torch.float64, device=dev), (n_parts, n))
    return S.crow_indices().to(torch.int64), S.col_indices().to(torch.int32)


def p0_restriction_device(owner, n_parts: int):
    """``p0_restriction`` on the device: a torch CSR ``(n_parts x n)`` with a unit
    entry at (owner[j], j), rows in DOF order (a stable sort of the owners)."""
    import torch

    dev = owner.device
    own = owner.to(torch.int64)
    n = own.numel()
    cols = torch.argsort(own, stable=True)
    ptr = torch.zeros(n_parts + 1, dtype=torch.int64, device=dev)
    ptr[1:] = torch.cumsum(torch.bincount(own, minlength=n_parts), 0)
    return torch.sparse_csr_tensor(ptr, cols, torch.ones(n, dtype=torch.float64, device=dev), (n_parts, n))


def q1_coarse_restriction_device(dim: int, n_el: int, parts_per_axis: int, device):
    """``q1_coarse_restriction`` on the device: every fine interior node takes the
    multilinear weights of the 2^dim coarse nodes around it (the zero weights and
    the Dirichlet coarse nodes dropped); the weights are multiplied slowest axis
    first, as the Kronecker product of the 1D interpolations does, so the entries
    are identical. Returns a torch CSR ``((parts_per_axis - 1)^dim x (n_el - 1)^dim)``
    with sorted columns."""
    import torch

    P_ax = parts_per_axis
    assert n_el % P_ax == 0
    H = n_el // P_ax
    m = n_el - 1
    mc = P_ax - 1
    # 1D: fine node p = 1..m -> (coarse index, weight) for its two neighbours
    p = torch.arange(1, m + 1, dtype=torch.int64, device=device)
    c0 = p // H
    t = (p - c0 * H).to(torch.float64) / H
    c1d = torch.stack([c0, c0 + 1], 1)                  # (m, 2)
    w1d = torch.stack([1.0 - t, t], 1)
    ok1d = (c1d >= 1) & (c1d <= mc) & (w1d != 0.0)
    n = m ** dim
    fine = torch.arange(n, dtype=torch.int64, device=device)
    # per axis (slowest first) the fine coordinate of every fine node
    coords = [(fine // (m ** (dim - 1 - a))) % m for a in range(dim)]
    combos = torch.cartesian_prod(*[torch.arange(2, device=device)] * dim).reshape(-1, dim)  # (2^dim, dim)
    rows, cols, vals = [], [], []
    for cmb in combos.tolist():
        w = None
        c = torch.zeros(n, dtype=torch.int64, device=device)
        ok = torch.ones(n, dtype=torch.bool, device=device)
        for a in range(dim):
            wa = w1d[coords[a], cmb[a]]
            w = wa if w is None else w * wa
            c = c * mc + (c1d[coords[a], cmb[a]] - 1)
            ok &= ok1d[coords[a], cmb[a]]
        rows.append(c[ok])
        cols.append(fine[ok])
        vals.append(w[ok])
    rows, cols, vals = torch.cat(rows), torch.cat(cols), torch.cat(vals)
    order = torch.argsort(rows * n + cols)
    rows, cols, vals = rows[order], cols[order], vals[order]
    n_c = mc ** dim
    ptr = torch.zeros(n_c + 1, dtype=torch.int64, device=device)
    ptr[1:] = torch.cumsum(torch.bincount(rows, minlength=n_c), 0)
    return torch.sparse_csr_tensor(ptr, cols, vals, (n_c, n))
