"""Sparse SPD direct solver for large coarse problems: nested dissection +
multifrontal Cholesky, applied by per-level GEMV kernels.

The reference factors its coarse matrix ``A_C = R0 A R0^T`` once with cuDSS
(``src/dd_solvers/dd_solvers/solvers.py:85-113``, ``cpp/cudss.cpp:64-105``) and
calls the cuDSS solve in every preconditioner application. Its experiments use
coarse spaces of 65k-1M DOFs (P0 on the ``S8``-``S10`` / ``C8``-``C10`` meshes),
far beyond a dense inverse. cuDSS is not in this image; this module is the
replacement for those sizes.

Setup (host symbolic phase, device numeric phase):

1. *Ordering.* Recursive vertex bisection of the matrix graph: a BFS from a
   pseudo-peripheral vertex, the median level set as the separator, each
   connected component handled on its own, down to leaves of at most
   ``leaf`` vertices. The separator tree in post-order is the elimination
   order (subtrees first, then their separator).
2. *Symbolic.* Front ``t`` holds its separator ``S_t`` followed by its update
   set ``U_t`` = the later-eliminated vertices coupled to the subtree
   (``adj(S_t)`` plus the children's update sets, restricted to ancestors).
3. *Numeric.* Level by level from the leaves, a padded batch of dense fronts
   is assembled from ``A`` and the children's update matrices (extend-add,
   one child slot at a time so no two additions meet), then
   ``L = chol(F_SS)``, ``Linv = L^-1``, ``M = F_US F_SS^-1`` and the update
   ``F_UU - F_US F_SS^-1 F_SU``. The stored operator of front ``t`` is
   ``G_t = [Linv; M]`` (``(s+u) x s``, row-major, FP64).

Solve (``ddx_coarse_solve_nd``, one forward launch and one backward launch per
tree level):

* forward, leaves to root: ``f = [w_S; 0] + sum of the children's update
  vectors`` (fixed order), ``y_S = Linv f_S``, ``u_t = f_U - M f_S``; on
  levels whose fronts are cut into many forward items, a gather launch
  assembles ``f`` once per front first (the items would otherwise each
  repeat the gather of ``f_S``);
* backward, root to leaves: ``x_S = Linv^T y_S - M^T x_U``.

Both are dense GEMVs over ``G_t``, split into row (forward) or column
(backward) chunks so that large fronts spread over many CTAs; every sum is in
a fixed order, so results are deterministic. The sweeps are latency-bound;
up to ``OVERLAP_MAX_N`` rows each item stages its operator rows in shared
memory before waiting on the previous level and releases the next level
right after that wait (measured on B200: -10% PCG time at 131k coarse rows,
-9% at 524k, no change at 1.05M; above 1M rows it stays off).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as L

LEAF = 128          # largest subgraph left undissected (a leaf front)
TOP_MERGE = 2048    # merge the top levels into one dense front while it holds at most this many vertices
ITEM_BYTES = 32768  # operator bytes per work item (rows of G or of G^T) ...
ITEM_MAX_ROWS = 64  # ... between 8 and this many rows
FAT_ITEMS_MIN_N = 1_000_000  # above this many rows: items of 64 KB and up to 128 rows
GATHER_POSITIONS = 256  # front positions per gather item
GATHER_MIN_RATIO = 2.0  # gather f once per front on levels whose items would gather >= this x its size
GATHER_MIN_LEVEL = 1    # ... from this tree level up (leaf fronts have no children to add)
# Latency hiding in the sweeps: operator rows staged in shared memory before
# the wait on the previous level (STAGE), the gather launches (GATHER) and the
# early release of the next level's kernel (RELEASE); all three for coarse
# problems of up to OVERLAP_MAX_N rows, and staging only on levels of at most
# STAGE_MAX_WAVES x (SMs x 4) items (None: every level).
OVERLAP_MAX_N = 1_000_000
STAGE, GATHER, RELEASE = True, True, True
STAGE_MAX_WAVES = None


def _rows_per_item(row_len, item_bytes: int, max_rows: int):
    """Rows of ``row_len`` doubles per work item: about ``item_bytes`` of
    operator, a multiple of 8 between 8 and ``max_rows`` (elementwise on arrays)."""
    r = item_bytes // (8 * np.maximum(row_len, 1))
    return np.minimum(max_rows, np.maximum(8, r // 8 * 8))


def _cut_items(levels, length, width, item_bytes: int, max_rows: int):
    """Work items (front, first row, rows) over the fronts of ``levels`` in
    order: front t's ``length[t]`` rows of ``width[t]`` doubles cut into runs
    of ``_rows_per_item(width[t])``. Returns the (k, 3) int32 items and the
    per-level item pointer."""
    sizes = np.array([len(f) for f in levels], dtype=np.int64)
    fronts = np.concatenate([np.asarray(f, dtype=np.int64) for f in levels] + [np.zeros(0, dtype=np.int64)])
    ln = np.maximum(length[fronts], 1)
    step = _rows_per_item(width[fronts], item_bytes, max_rows)
    count = -(-ln // step)
    ccum = np.concatenate([[0], np.cumsum(count)]).astype(np.int64)
    ptr = ccum[np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)]
    t = np.repeat(fronts, count)
    k = np.arange(int(count.sum())) - np.repeat(np.cumsum(count) - count, count)
    st = np.repeat(step, count)
    r0 = k * st
    nr = np.minimum(st, np.repeat(length[fronts], count) - r0)
    return np.stack([t, r0, nr], axis=1).astype(np.int32), ptr


# ---------------------------------------------------------------------------
# ordering
# ---------------------------------------------------------------------------

def nested_dissection(indptr: np.ndarray, indices: np.ndarray, n: int, leaf: int = 128):
    """Separator tree of the graph of an ``n x n`` symmetric pattern, from the
    native ``ddx_nd_order``. Returns ``(S, parent)`` in post-order: ``S[t]``
    the vertices node ``t`` eliminates, ``parent[t]`` its parent (-1: root)."""
    indptr = np.ascontiguousarray(indptr, dtype=np.int64)
    indices = np.ascontiguousarray(indices, dtype=np.int64)
    perm = np.empty(max(n, 1), dtype=np.int64)
    first = np.empty(n + 2, dtype=np.int64)
    parent = np.empty(n + 1, dtype=np.int64)
    count = np.zeros(1, dtype=np.int64)
    L.call("ddx_nd_order", n, indptr.ctypes.data, indices.ctypes.data, int(leaf), perm.ctypes.data,
           first.ctypes.data, parent.ctypes.data, count.ctypes.data)
    nf = int(count[0])
    S = [perm[first[t]:first[t + 1]].copy() for t in range(nf)]
    return S, parent[:nf].copy()


def _update_sets(n: int, s_first, s_size, p_ptr, p_pos, parent):
    """Update sets of the separator tree (``ddx_nd_update_sets``): CSR
    ``(u_ptr, u_pos)`` of elimination positions, front by front: the
    positions after the front's separator that its rows or its children's
    update sets reach, sorted and distinct."""
    a = [np.ascontiguousarray(x, dtype=np.int64) for x in (s_first, s_size, p_ptr, p_pos, parent)]
    nf = len(a[1])
    u_ptr = np.empty(nf + 1, dtype=np.int64)
    total = np.zeros(1, dtype=np.int64)
    cap = 2 * len(a[3]) + n
    for _ in range(2):
        u_pos = np.empty(max(cap, 1), dtype=np.int64)
        try:
            L.call("ddx_nd_update_sets", n, nf, *(x.ctypes.data for x in a), u_ptr.ctypes.data, u_pos.ctypes.data,
                   cap, total.ctypes.data)
            return u_ptr, u_pos[:int(total[0])]
        except L.DDXError:
            if int(total[0]) <= cap:
                raise
            cap = int(total[0])
    raise RuntimeError("ddx_nd_update_sets: capacity")


def _merge_top(S: list, parent: np.ndarray, limit: int):
    """Merge the top levels of the separator tree into one front while the
    merged separators hold at most ``limit`` vertices: whole levels, from the
    root(s) down. The other nodes keep their post-order (each remaining subtree
    stays contiguous), the merged front comes last, and the children of merged
    nodes become its children. Fewer levels means fewer latency-bound sweep
    launches; the merged front is one dense factor."""
    nf = len(S)
    if limit <= 0 or nf < 2:
        return S, parent
    children = [[] for _ in range(nf)]
    for t in range(nf):
        if parent[t] >= 0:
            children[parent[t]].append(t)
    depth = np.zeros(nf, dtype=np.int64)  # distance from the root
    for t in range(nf - 1, -1, -1):  # post-order: parents after children
        if parent[t] >= 0:
            depth[t] = depth[parent[t]] + 1
    sizes = np.array([len(x) for x in S], dtype=np.int64)
    top, total = None, 0
    for d in range(int(depth.max()) + 1):
        layer = np.nonzero(depth == d)[0]
        if total + int(sizes[layer].sum()) > limit:
            break
        total += int(sizes[layer].sum())
        top = d
    if top is None or top == 0 and len(np.nonzero(depth == 0)[0]) == nf:
        return S, parent
    merged = depth <= top
    keep = [t for t in range(nf) if not merged[t]]
    new_id = {t: i for i, t in enumerate(keep)}
    root = len(keep)
    S2 = [S[t] for t in keep] + [np.concatenate([S[t] for t in range(nf) if merged[t]])]
    parent2 = np.full(root + 1, -1, dtype=np.int64)
    for t in keep:
        p = parent[t]
        parent2[new_id[t]] = root if merged[p] else new_id[p]
    return S2, parent2


# ---------------------------------------------------------------------------
# symbolic analysis
# ---------------------------------------------------------------------------

class NDSymbolic:
    """Fronts in post-order with their index sets, levels and gather maps."""

    def __init__(self, indptr, indices, n: int, leaf: int = 128, top_merge: int | None = None):
        S, parent = nested_dissection(indptr, indices, n, leaf)
        S, parent = _merge_top(S, parent, TOP_MERGE if top_merge is None else top_merge)
        indptr = np.asarray(indptr, dtype=np.int64)
        indices = np.asarray(indices, dtype=np.int64)
        nf = len(S)
        children = [[] for _ in range(nf)]
        for t in range(nf):
            if parent[t] >= 0:
                children[parent[t]].append(t)
        perm = np.concatenate(S) if nf else np.zeros(0, dtype=np.int64)
        pos = np.empty(n, dtype=np.int64)
        pos[perm] = np.arange(n)
        s_sizes = np.array([len(x) for x in S], dtype=np.int64)
        s_first = np.concatenate([[0], np.cumsum(s_sizes)[:-1]])
        # the rows of A in elimination order: a front's separator rows are one slice
        deg = np.diff(indptr)[perm]
        p_ptr = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(deg, out=p_ptr[1:])
        p_idx = indices[np.repeat(indptr[perm] - p_ptr[:-1], deg) + np.arange(int(p_ptr[-1]))] if n else indices
        p_pos = pos[p_idx]
        u_ptr, u_pos = _update_sets(n, s_first, s_sizes, p_ptr, p_pos, parent)
        U = [perm[u_pos[u_ptr[t]:u_ptr[t + 1]]] for t in range(nf)]
        level = np.zeros(nf, dtype=np.int64)
        for t in range(nf):
            if children[t]:
                level[t] = 1 + max(level[c] for c in children[t])
        self.n, self.nf = n, nf
        self.S, self.U, self.children, self.parent = S, U, children, parent
        self.perm, self.pos = perm, pos
        self.level = level
        self.n_levels = int(level.max()) + 1 if nf else 0
        self.s = s_sizes
        self.u = np.array([len(x) for x in U], dtype=np.int64)
        m = self.s + self.u
        self.idx_off = np.concatenate([[0], np.cumsum(m)[:-1]]).astype(np.int64)
        self.g_off = np.concatenate([[0], np.cumsum(m * self.s)[:-1]]).astype(np.int64)
        self.upd_off = np.concatenate([[0], np.cumsum(self.u)[:-1]]).astype(np.int64)
        self.g_total = int((m * self.s).sum())
        self.upd_total = int(self.u.sum())
        self.fidx = np.concatenate([np.concatenate([S[t], U[t]]) for t in range(nf)]).astype(np.int64)
        # extend-add positions of each child's update set inside its parent's front:
        # one search over (front, elimination position) keys, sorted because each
        # front lists its separator and then its update set in elimination order
        assert (self.u[parent < 0] == 0).all(), "a root front with an update set"
        total = int(m.sum())
        front_of = np.repeat(np.arange(nf, dtype=np.int64), m)
        within = np.arange(total, dtype=np.int64) - np.repeat(self.idx_off, m)
        keys = front_of * (n + 1) + pos[self.fidx]
        upd_v = self.fidx[within >= np.repeat(self.s, m)]  # U[0], U[1], ... (update-buffer order)
        upd_front = np.repeat(np.arange(nf, dtype=np.int64), self.u)
        query = parent[upd_front].astype(np.int64) * (n + 1) + pos[upd_v]
        gp = np.searchsorted(keys, query)
        assert (gp < total).all() and np.array_equal(keys[np.minimum(gp, total - 1)], query), \
            "update set not inside the parent front"
        rel_all = gp - self.idx_off[parent[upd_front]] if gp.size else gp
        self.rel = [None] * nf
        for t in np.nonzero(parent >= 0)[0]:
            self.rel[t] = rel_all[self.upd_off[t]:self.upd_off[t] + self.u[t]]
        # gather map: per front position, the update-buffer entries to add (children in order)
        gs = np.arange(self.upd_total, dtype=np.int64)
        if gp.size:
            order = np.argsort(gp, kind="stable")
            gp, gs = gp[order], gs[order]
        else:
            gp = gs = np.zeros(0, dtype=np.int64)
        self.gptr = np.zeros(total + 1, dtype=np.int64)
        np.add.at(self.gptr, gp + 1, 1)
        self.gptr = np.cumsum(self.gptr)
        self.gsrc = gs.astype(np.int64)
        self.by_level = [np.nonzero(level == lv)[0] for lv in range(self.n_levels)]
        m_all = self.s + self.u
        self.fwd_level_smax = np.array([int(self.s[f].max()) if len(f) else 0 for f in self.by_level],
                                       dtype=np.int32)
        self.bwd_level_mmax = np.array([int(m_all[f].max()) if len(f) else 0 for f in self.by_level[::-1]],
                                       dtype=np.int32)
        self.build_items()

    def build_items(self, item_bytes: int = ITEM_BYTES, max_rows: int = ITEM_MAX_ROWS) -> None:
        """Per-level work items: (front, first row, rows) of G_t for the forward
        sweep (leaves first), of G_t^T for the backward sweep (root first)."""
        m = self.s + self.u
        self.fwd_items, self.fwd_level_ptr = _cut_items(self.by_level, m, self.s, item_bytes, max_rows)
        self.bwd_items, self.bwd_level_ptr = _cut_items(self.by_level[::-1], self.s, m, item_bytes, max_rows)
        # largest operator range of an item per level (bytes): staged in shared memory where it fits
        self.fwd_level_gmax = np.zeros(self.n_levels, dtype=np.int64)
        self.bwd_level_gmax = np.zeros(self.n_levels, dtype=np.int64)
        for ptr, items, width, gmax in ((self.fwd_level_ptr, self.fwd_items, self.s, self.fwd_level_gmax),
                                        (self.bwd_level_ptr, self.bwd_items, m, self.bwd_level_gmax)):
            for j in range(self.n_levels):
                a, b = ptr[j], ptr[j + 1]
                if b > a:
                    gmax[j] = int((items[a:b, 2].astype(np.int64) * width[items[a:b, 0]]).max()) * 8
        # gather items (front, first position, positions) of the levels where
        # the forward items together would gather f_S many times over
        gat = []
        self.gat_level_ptr = np.zeros(self.n_levels + 1, dtype=np.int64)
        for lv in range(self.n_levels):
            a, b = self.fwd_level_ptr[lv], self.fwd_level_ptr[lv + 1]
            fronts = self.by_level[lv]
            repeated = int(self.s[self.fwd_items[a:b, 0]].sum()) if b > a else 0
            once = int(m[fronts].sum())
            if lv >= GATHER_MIN_LEVEL and once and repeated >= GATHER_MIN_RATIO * once:
                for t in fronts:
                    for p0 in range(0, int(m[t]), GATHER_POSITIONS):
                        gat.append((t, p0, min(GATHER_POSITIONS, int(m[t]) - p0)))
            self.gat_level_ptr[lv + 1] = len(gat)
        self.gat_items = np.array(gat, dtype=np.int32).reshape(-1, 3)


# ---------------------------------------------------------------------------
# numeric factorisation (torch, any device)
# ---------------------------------------------------------------------------

def _pairs(lengths: np.ndarray):
    """All index pairs ``(g, a, b)`` with ``a, b < lengths[g]`` (row-major per g)."""
    lengths = np.asarray(lengths, dtype=np.int64)
    sq = lengths * lengths
    g = np.repeat(np.arange(len(lengths)), sq)
    start = np.cumsum(sq) - sq
    p = np.arange(int(sq.sum()), dtype=np.int64) - start[g]
    u = lengths[g]
    return g, p // u, p % u


def factorize(sym: NDSymbolic, indptr, indices, values, device, max_batch_bytes: int = 1 << 30):
    """The stored operators ``G_t = [Linv; M]`` of every front, concatenated,
    and their transposes (same offsets)."""
    indptr = np.asarray(indptr, dtype=np.int64)
    indices = np.asarray(indices, dtype=np.int64)
    vals = torch.as_tensor(np.asarray(values, dtype=np.float64)) if not isinstance(values, torch.Tensor) \
        else values.to(torch.float64)
    vals = vals.to(device)
    n, nf = sym.n, sym.nf
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(indptr))
    front_of = np.empty(n, dtype=np.int64)
    front_of[sym.perm] = np.repeat(np.arange(nf), sym.s)
    first = np.cumsum(sym.s) - sym.s  # position of each front's first separator vertex
    # original entries (i in S_t, j in S_t or U_t): kept where pos(j) >= first position of S_t
    t_of = front_of[rows]
    keep = sym.pos[indices] >= first[t_of]
    e_t = t_of[keep]
    e_j = indices[keep]
    e_v = np.nonzero(keep)[0]
    li = sym.pos[rows[keep]] - first[e_t]
    # local index of j: its place in front t's list [S_t, U_t] (sorted by position)
    key_all = np.repeat(np.arange(nf, dtype=np.int64), sym.s + sym.u) * (n + 1) + sym.pos[sym.fidx]
    lj = np.searchsorted(key_all, e_t * (n + 1) + sym.pos[e_j]) - sym.idx_off[e_t]
    in_s = lj < sym.s[e_t]

    G = torch.zeros(sym.g_total, dtype=torch.float64, device=device)
    GT = torch.zeros(sym.g_total, dtype=torch.float64, device=device)
    upd = {}  # front -> (batch tensor, batch index) of its pending update matrix
    for lv in range(sym.n_levels):
        fronts = sym.by_level[lv]
        # chunk the level so a padded batch stays within max_batch_bytes
        sz = sym.s[fronts] + sym.u[fronts]
        chunks, cur, cur_max = [], [], 0
        for t, z in zip(fronts, sz):
            mm = max(cur_max, int(z))
            if cur and (len(cur) + 1) * (mm + 1) ** 2 * 8 > max_batch_bytes:
                chunks.append(cur)
                cur, mm = [], int(z)
            cur.append(int(t))
            cur_max = mm
        if cur:
            chunks.append(cur)
        for ch in chunks:
            ch = np.array(ch, dtype=np.int64)
            B = len(ch)
            sc, uc = sym.s[ch], sym.u[ch]
            SM, UM = int(sc.max()), int(uc.max())
            m = SM + UM
            F = torch.zeros(B, m, m, dtype=torch.float64, device=device)
            # identity on the padded separator diagonal
            npad = SM - sc
            if npad.any():
                pb = np.repeat(np.arange(B), npad)
                pi = np.arange(int(npad.sum())) - np.repeat(np.cumsum(npad) - npad, npad) + np.repeat(sc, npad)
                F[torch.as_tensor(pb, device=device), torch.as_tensor(pi, device=device),
                  torch.as_tensor(pi, device=device)] = 1.0
            # original entries (F_SS and F_US, mirrored into F_SU)
            bmap = np.full(nf, -1, dtype=np.int64)
            bmap[ch] = np.arange(B)
            sel = np.nonzero(bmap[e_t] >= 0)[0]
            if len(sel):
                et = e_t[sel]
                bb = torch.as_tensor(bmap[et], device=device)
                rt = torch.as_tensor(li[sel], device=device)
                c = lj[sel]
                ct = torch.as_tensor(np.where(in_s[sel], c, SM + (c - sym.s[et])), device=device)
                vv = vals[torch.as_tensor(e_v[sel], device=device)]
                F[bb, rt, ct] = vv
                us = torch.as_tensor(~in_s[sel], device=device)
                F[bb[us], ct[us], rt[us]] = vv[us]
            # extend-add of the children's updates, one child slot at a time
            nslots = max((len(sym.children[t]) for t in ch), default=0)
            for slot in range(nslots):
                groups = {}
                for b, t in enumerate(ch):
                    if slot < len(sym.children[t]):
                        c = sym.children[t][slot]
                        Ub, ub_i = upd.pop(c)
                        groups.setdefault(id(Ub), (Ub, []))[1].append((b, t, c, ub_i))
                for Ub, items in groups.values():
                    it = np.array(items, dtype=np.int64).reshape(-1, 4)
                    ucs = sym.u[it[:, 2]]
                    if not ucs.any():
                        continue
                    g, a, bq = _pairs(ucs)
                    rel = np.concatenate([sym.rel[c] for c in it[:, 2]])
                    rs = np.cumsum(ucs) - ucs
                    s_par = np.repeat(sym.s[it[:, 1]], ucs)
                    rel_pad = np.where(rel < s_par, rel, SM + (rel - s_par))
                    dst = it[g, 0] * m * m + rel_pad[rs[g] + a] * m + rel_pad[rs[g] + bq]
                    um = Ub.shape[1]
                    src = it[g, 3] * um * um + a * um + bq
                    F.view(-1).index_put_((torch.as_tensor(dst, device=device),),
                                          Ub.reshape(-1)[torch.as_tensor(src, device=device)], accumulate=True)
            Lc, info = torch.linalg.cholesky_ex(F[:, :SM, :SM])
            if int(info.abs().max()) != 0:
                raise RuntimeError("coarse matrix is not positive definite")
            eye = torch.eye(SM, dtype=torch.float64, device=device).expand(B, SM, SM)
            Linv = torch.linalg.solve_triangular(Lc, eye, upper=False)
            del Lc, eye
            if UM:
                W = F[:, SM:, :SM] @ Linv.transpose(1, 2)
                M = W @ Linv
                Upd = F[:, SM:, SM:] - W @ W.transpose(1, 2)
                del W
            else:
                M = Upd = None
            del F
            # store G_t = [Linv; M] (unpadded, row-major), one gather per chunk
            dev_s = torch.as_tensor(sc, device=device)
            dev_u = torch.as_tensor(uc, device=device)
            cnt = (dev_s + dev_u) * dev_s
            gb = torch.repeat_interleave(torch.arange(B, device=device), cnt)
            e = torch.arange(int(cnt.sum()), device=device) - torch.repeat_interleave(torch.cumsum(cnt, 0) - cnt, cnt)
            sb = dev_s[gb]
            row, col = e // sb, e % sb
            goff = torch.as_tensor(sym.g_off[ch], device=device)[gb]
            dst = goff + e
            dstT = goff + col * (sb + dev_u[gb]) + row  # (col, row) of the s x (s+u) transpose
            top = row < sb
            vtop = Linv.reshape(-1)[(gb * SM * SM + row * SM + col)[top]]
            G[dst[top]] = vtop
            GT[dstT[top]] = vtop
            if M is not None:
                bot = ~top
                vbot = M.reshape(-1)[(gb * UM * SM + (row - sb) * SM + col)[bot]]
                G[dst[bot]] = vbot
                GT[dstT[bot]] = vbot
            del gb, e, sb, row, col, dst, dstT, goff, top
            if Upd is not None:
                for b, t in enumerate(ch):
                    if sym.parent[t] >= 0:
                        upd[int(t)] = (Upd, b)
            del Linv, M
    return G, GT


# ---------------------------------------------------------------------------
# the plan handed to the kernels
# ---------------------------------------------------------------------------

class _Plan(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int), ("n_fronts", ctypes.c_int), ("n_levels", ctypes.c_int),
        ("max_front", ctypes.c_int),
        ("fwd_level_ptr", ctypes.c_void_p), ("bwd_level_ptr", ctypes.c_void_p),
        ("fwd_level_smax", ctypes.c_void_p), ("bwd_level_mmax", ctypes.c_void_p),
        ("fwd_items", ctypes.c_void_p), ("bwd_items", ctypes.c_void_p),
        ("front_s", ctypes.c_void_p), ("front_u", ctypes.c_void_p),
        ("g_off", ctypes.c_void_p), ("idx_off", ctypes.c_void_p), ("upd_off", ctypes.c_void_p),
        ("fidx", ctypes.c_void_p), ("gptr", ctypes.c_void_p), ("gsrc", ctypes.c_void_p),
        ("G", ctypes.c_void_p), ("GT", ctypes.c_void_p),
        ("s_first", ctypes.c_void_p), ("fpos", ctypes.c_void_p),
        ("gat_level_ptr", ctypes.c_void_p), ("gat_items", ctypes.c_void_p),
        ("fwd_level_gmax", ctypes.c_void_p), ("bwd_level_gmax", ctypes.c_void_p),
        ("release_early", ctypes.c_int),
    ]


class NDSolver:
    """Factor once (``A`` a torch CSR tensor on the device, FP64), then
    ``solve_into(w, x, R)`` with ``w, x`` (n, R) row-major FP64 on the device."""

    def __init__(self, A: torch.Tensor, leaf: int | None = None, top_merge: int | None = None):
        leaf = LEAF if leaf is None else leaf
        dev = A.device
        self.leaf = leaf
        indptr = A.crow_indices().cpu().numpy()
        indices = A.col_indices().cpu().numpy()
        self.n = A.shape[0]
        self.sym = sym = NDSymbolic(indptr, indices, self.n, leaf, top_merge)
        self.G, self.GT = factorize(sym, indptr, indices, A.values(), dev)
        i32 = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.int32, device=dev)  # noqa: E731
        i64 = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.int64, device=dev)  # noqa: E731
        self.t = {
            "front_s": i32(sym.s), "front_u": i32(sym.u),
            "g_off": i64(sym.g_off), "idx_off": i64(sym.idx_off), "upd_off": i64(sym.upd_off),
            "fidx": i32(sym.fidx), "gptr": i64(sym.gptr), "gsrc": i64(sym.gsrc),
            "s_first": i64(np.cumsum(sym.s) - sym.s), "fpos": i32(sym.pos[sym.fidx]),
        }
        self.fwd_level_smax = np.ascontiguousarray(sym.fwd_level_smax, dtype=np.int32)
        self.bwd_level_mmax = np.ascontiguousarray(sym.bwd_level_mmax, dtype=np.int32)
        self.max_front = int((sym.s + sym.u).max()) if sym.nf else 0
        p = _Plan()
        p.n, p.n_fronts, p.n_levels, p.max_front = self.n, sym.nf, sym.n_levels, self.max_front
        p.fwd_level_smax = self.fwd_level_smax.ctypes.data
        p.bwd_level_mmax = self.bwd_level_mmax.ctypes.data
        for k, v in self.t.items():
            setattr(p, k, v.data_ptr())
        p.G = self.G.data_ptr()
        p.GT = self.GT.data_ptr()
        self.plan = p
        if self.n > FAT_ITEMS_MIN_N:
            # measured on B200 (hybrid FP16 PCG, same box): with staging, 32 KB items are 9% faster at 524k
            # coarse rows, equal at 1.05M; unstaged 64 KB items are 1% faster at 2.1M
            sym.build_items(65536, 128)
        self._set_items()
        self._work = {}
        self.factor_bytes = 2 * self.G.numel() * 8

    def _set_items(self) -> None:
        sym, dev, p = self.sym, self.G.device, self.plan
        self.t["fwd_items"] = torch.as_tensor(sym.fwd_items.reshape(-1), dtype=torch.int32, device=dev)
        self.t["bwd_items"] = torch.as_tensor(sym.bwd_items.reshape(-1), dtype=torch.int32, device=dev)
        self.fwd_level_ptr = np.ascontiguousarray(sym.fwd_level_ptr, dtype=np.int64)
        self.bwd_level_ptr = np.ascontiguousarray(sym.bwd_level_ptr, dtype=np.int64)
        p.fwd_items = self.t["fwd_items"].data_ptr()
        p.bwd_items = self.t["bwd_items"].data_ptr()
        p.fwd_level_ptr = self.fwd_level_ptr.ctypes.data
        p.bwd_level_ptr = self.bwd_level_ptr.ctypes.data
        self.t["gat_items"] = torch.as_tensor(sym.gat_items.reshape(-1), dtype=torch.int32, device=dev)
        self.gat_level_ptr = np.ascontiguousarray(sym.gat_level_ptr, dtype=np.int64)
        p.gat_items = self.t["gat_items"].data_ptr()
        p.gat_level_ptr = self.gat_level_ptr.ctypes.data
        overlap = self.n <= OVERLAP_MAX_N
        fg = np.ascontiguousarray(sym.fwd_level_gmax, dtype=np.int64).copy()
        bg = np.ascontiguousarray(sym.bwd_level_gmax, dtype=np.int64).copy()
        if not (overlap and STAGE):
            fg[:] = -1
            bg[:] = -1
        elif STAGE_MAX_WAVES is not None:
            sms = torch.cuda.get_device_properties(dev).multi_processor_count if dev.type == "cuda" else 148
            limit = STAGE_MAX_WAVES * sms * 4
            fg[np.diff(sym.fwd_level_ptr) > limit] = -1
            bg[np.diff(sym.bwd_level_ptr) > limit] = -1
        self.fwd_level_gmax, self.bwd_level_gmax = fg, bg
        p.fwd_level_gmax = fg.ctypes.data
        p.bwd_level_gmax = bg.ctypes.data
        p.release_early = int(overlap and RELEASE)
        self.gather = overlap and GATHER

    def set_items(self, item_bytes: int, max_rows: int) -> None:
        """Re-cut the work items (a tuning knob: bytes of operator per CTA)."""
        self.sym.build_items(item_bytes, max_rows)
        self._set_items()

    def workspace(self, R: int, device):
        w = self._work.get(R)
        if w is None or (self.gather and w["fb"] is None):
            w = {"y": torch.empty(self.n * R, dtype=torch.float64, device=device),
                 "xe": torch.empty(self.n * R, dtype=torch.float64, device=device),
                 "upd": torch.empty(max(self.sym.upd_total, 1) * R, dtype=torch.float64, device=device),
                 "fb": torch.empty(max(len(self.sym.fidx), 1) * R, dtype=torch.float64, device=device)
                 if self.gather else None}
            self._work[R] = w
        return w

    def solve_into(self, w: torch.Tensor, x: torch.Tensor, R: int, ist=None) -> None:
        ws = self.workspace(R, w.device)
        L.call("ddx_coarse_solve_nd", ctypes.addressof(self.plan), R, L.ptr(w), L.ptr(x), L.ptr(ws["y"]),
               L.ptr(ws["xe"]), L.ptr(ws["upd"]), L.ptr(ws["fb"] if self.gather else None), L.ptr(ist),
               L.stream_ptr())

    def solve(self, rhs: torch.Tensor) -> torch.Tensor:
        L.require_cuda(rhs, "rhs")
        R = 1 if rhs.dim() == 1 else rhs.shape[1]
        w = rhs.to(torch.float64).contiguous()
        x = torch.empty_like(w)
        self.solve_into(w, x, R)
        return x.to(rhs.dtype)
