"""Seeded synthetic elliptic FEM problems (host-side setup, not on the solve path).

The reference builds its systems with DOLFINx (symmetric interior-penalty DG,
``src/experiments/experiments/discretization.py:32-96``). The workloads this
package is measured on are continuous finite elements instead, so the
assemblers live here:

* ``q1_grid``      - Q1 (bi/trilinear) elements on a uniform ``N^d`` grid of the
                     unit square/cube, per-element coefficient kappa, homogeneous
                     Dirichlet nodes eliminated. Assembled directly in stencil
                     form (9-point in 2D, 27-point in 3D), so the CSR rows come
                     out with sorted column indices and no COO sort is needed.
* ``p1_jittered``  - P1 triangles on a node grid whose interior nodes are
                     jittered by +-``jitter*h`` (two triangles per cell, one
                     diagonal direction), kappa per triangle (7-point pattern).
* ``gaussian_random_field`` - squared-exponential Gaussian field on a grid by
                     circulant embedding (FFT), seeded.

All matrices are ``scipy.sparse.csr_matrix`` in FP64 with int32 indices.
Interior DOFs are numbered lexicographically with x fastest.
"""
from __future__ import annotations

import dataclasses
import itertools

import numpy as np
import scipy.sparse as sps


@dataclasses.dataclass
class GridProblem:
    """A discretised problem on a structured (possibly jittered) grid.

    ``matrix`` is SPD on the interior DOFs; ``dim`` and ``n_el`` describe the
    element grid (``n_el`` elements per axis); ``interior_shape`` is the
    per-axis count of interior nodes (x fastest in the DOF numbering);
    ``coords`` are the DOF coordinates (n, dim); ``mass`` is the lumped mass
    per DOF (used to turn a nodal source f into a load vector).
    """

    matrix: sps.csr_matrix
    dim: int
    n_el: int
    interior_shape: tuple
    coords: np.ndarray
    mass: np.ndarray
    kappa: np.ndarray | None = None
    kind: str = "q1"
    # For P1: triangle -> node (global node grid ids) and geometry, used by the
    # element-gradient kernel setup.
    elements: np.ndarray | None = None


def _gauss_1d():
    g = 1.0 / np.sqrt(3.0)
    return np.array([-g, g]) * 0.5 + 0.5, np.array([0.5, 0.5])


def q1_reference_stiffness(dim: int) -> np.ndarray:
    """Stiffness of the unit reference cell for Q1 with unit coefficient.

    Local node ``a`` has bit ``d`` of ``a`` equal to its coordinate along axis
    ``d``. Integrated exactly with the 2-point Gauss rule per axis.
    Scaling to a cell of side h multiplies by ``h**(dim-2)``.
    """
    pts, wts = _gauss_1d()
    nloc = 2 ** dim
    K = np.zeros((nloc, nloc))
    for q in itertools.product(range(2), repeat=dim):
        xq = np.array([pts[i] for i in q])
        wq = np.prod([wts[i] for i in q])
        grads = np.zeros((nloc, dim))
        for a in range(nloc):
            bits = [(a >> d) & 1 for d in range(dim)]
            for d in range(dim):
                g = 1.0
                for e in range(dim):
                    phi_e = xq[e] if bits[e] else 1.0 - xq[e]
                    dphi_e = 1.0 if bits[e] else -1.0
                    g *= dphi_e if e == d else phi_e
                grads[a, d] = g
        K += wq * grads @ grads.T
    return K


def q1_grid(dim: int, n_el: int, kappa: np.ndarray | None = None) -> GridProblem:
    """Q1 stiffness on ``n_el**dim`` cells of the unit square/cube.

    ``kappa`` has shape ``(n_el,)*dim`` indexed ``[ez, ey, ex]`` (3D) or
    ``[ey, ex]`` (2D); ``None`` means kappa = 1. Boundary nodes carry
    homogeneous Dirichlet values and are eliminated.
    """
    assert dim in (2, 3)
    m = n_el - 1  # interior nodes per axis
    h = 1.0 / n_el
    if kappa is None:
        kappa = np.ones((n_el,) * dim)
    kappa = np.asarray(kappa, dtype=np.float64)
    assert kappa.shape == (n_el,) * dim
    Kref = q1_reference_stiffness(dim) * h ** (dim - 2)

    # Interior node multi-index arrays, axis order (z, y, x) with x fastest.
    n = m ** dim
    offsets = list(itertools.product((-1, 0, 1), repeat=dim))  # sorted -> column order
    vals = np.zeros((len(offsets),) + (m,) * dim)
    # Node p (interior, 1-based grid coordinates) and neighbour p+o share the
    # cells c with c_d in {p_d-1, p_d} and c_d in {p_d+o_d-1, p_d+o_d}.
    for oi, off in enumerate(offsets):
        # per axis, the admissible cell shifts s (cell index = p_d - 1 + s, s in {0,1})
        choices = []
        for o in off:
            choices.append([s for s in (0, 1) if s - o in (0, 1)])
        for shifts in itertools.product(*choices):
            # local index of node p in cell: (1 - s); of neighbour: (1 - s + o)
            la = 0
            lb = 0
            for d in range(dim):
                # axis d in (z,y,x) order corresponds to bit (dim-1-d)
                bit = dim - 1 - d
                la |= (1 - shifts[d]) << bit
                lb |= (1 - shifts[d] + off[d]) << bit
            coef = Kref[la, lb]
            # cells indexed [p_d - 1 + s_d] for p_d in 1..m  -> slice s_d : s_d + m
            sl = tuple(slice(shifts[d], shifts[d] + m) for d in range(dim))
            vals[oi] += coef * kappa[sl]
    # Validity mask (neighbour interior) and column ids.
    grids = np.meshgrid(*[np.arange(m)] * dim, indexing="ij")  # (z,y,x)
    cols = np.empty((len(offsets), n), dtype=np.int64)
    valid = np.empty((len(offsets), n), dtype=bool)
    for oi, off in enumerate(offsets):
        ok = np.ones((m,) * dim, dtype=bool)
        lin = np.zeros((m,) * dim, dtype=np.int64)
        for d in range(dim):
            q = grids[d] + off[d]
            ok &= (q >= 0) & (q < m)
            lin = lin * m + q
        valid[oi] = ok.ravel()
        cols[oi] = lin.ravel()
    valid_t = valid.T  # (n, noff)
    counts = valid_t.sum(axis=1)
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=indptr[1:])
    indices = cols.T[valid_t].astype(np.int32)
    data = vals.reshape(len(offsets), n).T[valid_t]
    A = sps.csr_matrix((data, indices, indptr.astype(np.int32)), shape=(n, n))
    A.has_sorted_indices = True

    ax = (np.arange(m) + 1) * h
    mesh = np.meshgrid(*[ax] * dim, indexing="ij")
    coords = np.stack([g.ravel() for g in reversed(mesh)], axis=1)  # (x, y[, z])
    mass = np.full(n, h ** dim)
    return GridProblem(A, dim, n_el, (m,) * dim, coords, mass, kappa, "q1")


def p1_jittered(n_nodes: int, jitter: float, kappa_sigma: float, seed: int) -> GridProblem:
    """P1 triangles on an ``n_nodes x n_nodes`` node grid of the unit square.

    Interior nodes move by i.i.d. uniform offsets in ``[-jitter*h, jitter*h]``
    per coordinate; each cell is split along its (0,0)-(1,1) diagonal. The
    per-triangle coefficient is log-normal ``exp(sigma * N(0,1))``. Boundary
    nodes are Dirichlet and eliminated, so there are ``(n_nodes-2)**2`` DOFs.
    Random draws, in order: x jitter, y jitter (interior nodes), triangle
    log-coefficients (lower triangles then upper, cell-major).
    """
    rng = np.random.default_rng(seed)
    N = n_nodes
    h = 1.0 / (N - 1)
    X, Y = np.meshgrid(np.arange(N) * h, np.arange(N) * h, indexing="xy")  # [j, i]
    m = N - 2
    X[1:-1, 1:-1] += rng.uniform(-jitter * h, jitter * h, size=(m, m))
    Y[1:-1, 1:-1] += rng.uniform(-jitter * h, jitter * h, size=(m, m))
    ncell = N - 1
    g = rng.standard_normal((2, ncell, ncell))
    kap = np.exp(kappa_sigma * g)

    # Triangle types in cell (i, j) with corners c00=(j,i), c10=(j,i+1), c11, c01:
    #   lower: c00, c10, c11  ; upper: c00, c11, c01
    tri_types = [((0, 0), (0, 1), (1, 1)), ((0, 0), (1, 1), (1, 0))]  # (dj, di)
    offs = [(-1, -1), (-1, 0), (0, -1), (0, 0), (0, 1), (1, 0), (1, 1)]  # (dj, di) sorted
    off_id = {o: k for k, o in enumerate(offs)}
    vals = np.zeros((len(offs), N, N))
    elements = []
    for t, corners in enumerate(tri_types):
        P = [(X[dj:dj + ncell, di:di + ncell], Y[dj:dj + ncell, di:di + ncell]) for dj, di in corners]
        (x0, y0), (x1, y1), (x2, y2) = P
        det = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0)
        area = 0.5 * np.abs(det)
        # gradients of barycentric basis functions
        gx = [(y1 - y2) / det, (y2 - y0) / det, (y0 - y1) / det]
        gy = [(x2 - x1) / det, (x0 - x2) / det, (x1 - x0) / det]
        ke = kap[t] * area
        for a in range(3):
            for b in range(3):
                coef = ke * (gx[a] * gx[b] + gy[a] * gy[b])
                (dja, dia), (djb, dib) = corners[a], corners[b]
                o = off_id[(djb - dja, dib - dia)]
                vals[o, dja:dja + ncell, dia:dia + ncell] += coef
        elements.append(corners)
    # Restrict to interior rows/cols.
    n = m * m
    jj, ii = np.meshgrid(np.arange(1, N - 1), np.arange(1, N - 1), indexing="ij")
    cols = np.empty((len(offs), n), dtype=np.int64)
    valid = np.empty((len(offs), n), dtype=bool)
    data = np.empty((len(offs), n))
    for k, (dj, di) in enumerate(offs):
        qj, qi = jj + dj, ii + di
        ok = (qj >= 1) & (qj <= N - 2) & (qi >= 1) & (qi <= N - 2)
        valid[k] = ok.ravel()
        cols[k] = ((qj - 1) * m + (qi - 1)).ravel()
        data[k] = vals[k, 1:-1, 1:-1].ravel()
    vt = valid.T
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(vt.sum(axis=1), out=indptr[1:])
    A = sps.csr_matrix((data.T[vt], cols.T[vt].astype(np.int32), indptr.astype(np.int32)), shape=(n, n))
    A.has_sorted_indices = True
    coords = np.stack([X[1:-1, 1:-1].ravel(), Y[1:-1, 1:-1].ravel()], axis=1)
    # lumped mass: one third of the adjacent triangle areas
    mass_full = np.zeros((N, N))
    for t, corners in enumerate(tri_types):
        P = [(X[dj:dj + ncell, di:di + ncell], Y[dj:dj + ncell, di:di + ncell]) for dj, di in corners]
        (x0, y0), (x1, y1), (x2, y2) = P
        area = 0.5 * np.abs((x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0))
        for dj, di in corners:
            mass_full[dj:dj + ncell, di:di + ncell] += area / 3.0
    mass = mass_full[1:-1, 1:-1].ravel()
    return GridProblem(A, 2, N - 1, (m, m), coords, mass, kap, "p1")


def gaussian_random_field(n: int, length_scale: float, seed: int, dim: int = 2) -> np.ndarray:
    """Stationary Gaussian field with squared-exponential covariance on a grid.

    Values at the ``n**dim`` cell centres of the unit square/cube, unit
    variance, covariance ``exp(-|x-y|^2 / (2 l^2))``. Sampled exactly by
    circulant embedding on a periodic grid of ``2n`` points per axis (period
    2, larger than the support needed for l = 0.1); negative eigenvalues of
    the embedding (round-off size) are clipped to zero. One complex normal
    draw gives the field as its real part.
    """
    rng = np.random.default_rng(seed)
    M = 2 * n
    h = 1.0 / n
    d1 = np.minimum(np.arange(M), M - np.arange(M)) * h
    grids = np.meshgrid(*[d1] * dim, indexing="ij")
    r2 = sum(g * g for g in grids)
    c = np.exp(-r2 / (2.0 * length_scale ** 2))
    lam = np.fft.fftn(c).real
    lam = np.maximum(lam, 0.0)
    xi = rng.standard_normal((M,) * dim) + 1j * rng.standard_normal((M,) * dim)
    f = np.fft.fftn(np.sqrt(lam / lam.size) * xi)
    sl = tuple(slice(0, n) for _ in range(dim))
    return np.ascontiguousarray(f.real[sl])


def uniform_rhs(n: int, seed: int, nrhs: int | None = None) -> np.ndarray:
    """Load vector with i.i.d. uniform[-1, 1] entries (the reference's
    ``random_rhs`` mode, ``src/experiments/experiments/experiments.py:242-245``)."""
    rng = np.random.default_rng(seed)
    shape = (n,) if nrhs is None else (n, nrhs)
    return rng.uniform(-1.0, 1.0, size=shape)


def normal_rhs(n: int, seed: int, nrhs: int | None = None) -> np.ndarray:
    rng = np.random.default_rng(seed)
    shape = (n,) if nrhs is None else (n, nrhs)
    return rng.standard_normal(shape)


# ---------------------------------------------------------------------------
# Named workloads (sizes as quoted for the measured configurations)
# ---------------------------------------------------------------------------

def poisson2d(n_el: int) -> GridProblem:
    return q1_grid(2, n_el)


def diffusion3d_lognormal(n_el: int, seed: int) -> GridProblem:
    """3D Q1 with kappa = exp(g), g i.i.d. N(0,1) per element."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((n_el,) * 3)
    return q1_grid(3, n_el, np.exp(g))


# ---------------------------------------------------------------------------
# DG block structure (the reference's BSR benchmark meshes)
# ---------------------------------------------------------------------------

def dg_block_size(dim: int, p: int) -> int:
    """DOFs per element of a P_p DG space on triangles (dim 2) or tetrahedra (dim 3)."""
    return (p + 1) * (p + 2) // 2 if dim == 2 else (p + 1) * (p + 2) * (p + 3) // 6


def dg_bsr_pattern_2d(n: int) -> tuple[np.ndarray, np.ndarray]:
    """Block sparsity of a DG operator on the 2 n^2 triangles of an n x n grid of
    squares, each cut by its (i, j)-(i+1, j+1) diagonal: block row e holds e
    and its face neighbours (up to 3), column indices sorted. Triangle 2 (j n + i)
    is the lower-right one of square (i, j), 2 (j n + i) + 1 the upper-left one;
    lower-right (i, j) borders upper-left (i, j), (i, j - 1) and (i + 1, j).
    Returns (crow, col) as int32.
    """
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="xy")
    i, j = i.ravel(), j.ravel()
    sq = j * n + i
    lo, up = 2 * sq, 2 * sq + 1
    rows, cols = [lo, up], [lo, up]  # diagonal blocks
    pairs = [(lo, up, np.ones_like(i, dtype=bool))]  # own diagonal
    m = j > 0
    pairs.append((lo[m], 2 * ((j[m] - 1) * n + i[m]) + 1, None))  # bottom edge
    m = i < n - 1
    pairs.append((lo[m], 2 * (j[m] * n + i[m] + 1) + 1, None))  # right edge
    for a, b, _ in pairs:
        rows += [a, b]
        cols += [b, a]
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    order = np.lexsort((c, r))
    r, c = r[order], c[order]
    crow = np.zeros(2 * n * n + 1, dtype=np.int64)
    np.add.at(crow, r + 1, 1)
    return np.cumsum(crow).astype(np.int32), c.astype(np.int32)


def dg_bsr_pattern_3d(n: int, device="cpu") -> tuple[np.ndarray, np.ndarray]:
    """Block sparsity of a DG operator on the 6 n^3 tetrahedra of an n^3 grid
    of cubes, each cut into the 6 tetrahedra along its (0,0,0)-(1,1,1)
    diagonal (tetrahedron (cube, p) = {v000, v000 + e_a, v000 + e_a + e_b,
    v111} for the p-th permutation (a, b, c) of the axes): block row t holds
    t and the tetrahedra sharing a face with it (up to 4), columns sorted.
    Faces are matched by sorting their vertex triples (on ``device``).
    Returns (crow, col) as int32.
    """
    import torch

    dev = torch.device(device)
    m = n + 1
    c = torch.arange(n ** 3, device=dev, dtype=torch.int64)
    ci, cj, ck = c % n, (c // n) % n, c // (n * n)
    base = (ck * m + cj) * m + ci
    step = {0: 1, 1: m, 2: m * m}
    perms = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
    tets = []
    for a, b, _ in perms:
        v0 = base
        v1 = base + step[a]
        v2 = v1 + step[b]
        v3 = base + 1 + m + m * m
        tets.append(torch.stack([v0, v1, v2, v3], dim=1))
    T = torch.stack(tets, dim=1).reshape(-1, 4)  # tet id = 6 cube + p
    nt = T.shape[0]
    faces = torch.cat([T[:, [1, 2, 3]], T[:, [0, 2, 3]], T[:, [0, 1, 3]], T[:, [0, 1, 2]]], dim=0)
    owner = torch.arange(nt, device=dev).repeat(4)
    faces, _ = torch.sort(faces, dim=1)
    k1 = faces[:, 0] * (m ** 3) + faces[:, 1]
    k2 = faces[:, 2]
    o = torch.sort(k2, stable=True).indices
    o = o[torch.sort(k1[o], stable=True).indices]  # lexicographic (k1, k2)
    k1, k2, owner = k1[o], k2[o], owner[o]
    same = (k1[1:] == k1[:-1]) & (k2[1:] == k2[:-1])
    a_, b_ = owner[:-1][same], owner[1:][same]
    rows = torch.cat([torch.arange(nt, device=dev), a_, b_])
    cols = torch.cat([torch.arange(nt, device=dev), b_, a_])
    key = rows * nt + cols
    key = torch.sort(key).values
    rows, cols = key // nt, key % nt
    crow = torch.zeros(nt + 1, dtype=torch.int64, device=dev)
    crow[1:] = torch.cumsum(torch.bincount(rows, minlength=nt), 0)
    return crow.cpu().numpy().astype(np.int32), cols.cpu().numpy().astype(np.int32)
