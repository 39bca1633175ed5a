"""Domain-sharded two-level Schwarz PCG: the subdomains split over ranks (one
process per GPU), each rank holding its own rows of every vector.

The reference runs ``CG.solve`` with ``AdditiveSchwarz`` / ``HybridSchwarz``
on one GPU (``src/dd_solvers/dd_solvers/solvers.py:228-297, 811-826,
874-888``). Sharded, every step of that loop keeps its arithmetic and gains one
exchange where the data crosses a shard boundary:

* parts (the non-overlapping owners the subdomains grow from) go to ranks in
  contiguous runs of about equal DOF counts; a rank owns the DOFs of its parts
  and the subdomains grown from them;
* each rank numbers its owned DOFs first (ascending global id), then its ghosts
  (DOFs its matrix rows or subdomains touch but another rank owns), sorted by
  owning rank, so the ghosts of one neighbour are one contiguous slice;
* ``q = A p``: the ghost rows of p come from their owners (halo exchange), then
  the local rows of A (owned rows, local columns) run through the SpMV kernel;
* ``z = M r``: the ghost rows of r come in by the same halo exchange; the local
  subdomains' products land in ``ylocal``; the rows of ``ylocal`` that belong
  to another rank's DOFs go to that rank (reverse exchange) and are appended to
  its ``ylocal``; every owned DOF then sums its entries, local and received, in
  ascending global subdomain order (the order of the one-GPU combine);
* coarse space: each rank restricts its owned columns (``R0[:, own] r`` or
  ``(R0 A)[:, own] y``), one all-reduce sums the coarse vector, and every rank
  solves the (replicated) coarse problem;
* PCG scalars: every fused reduction parks its per-rank column totals
  (``DDX_G_DEFER``), one all-reduce of 2R doubles sums them, and
  ``ddx_pcg_finalize`` runs the same step-length / stop-test epilogue on every
  rank, so all ranks take the same decisions.

``Comm`` carries the exchanges: ``DistComm`` over ``torch.distributed`` (NCCL
on GPUs, gloo on CPU) for one shard per process, ``LocalComm`` for all shards
in one process (copies and sums in rank order; on one GPU no kernel ever waits
for another shard, so the emulation is safe to run).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sps
import torch

__all__ = ["ShardPlan", "plan_shards", "part_ranks", "DistComm", "LocalComm", "ShardLinks", "halo_exchange",
           "reverse_exchange", "ShardedCG"]


# ---------------------------------------------------------------------------
# host plan
# ---------------------------------------------------------------------------

def part_ranks(owner: np.ndarray, n_parts: int, world: int) -> np.ndarray:
    """Rank of every part: contiguous runs of parts with about equal owned DOF
    counts (the cut after the part where the running count first reaches
    g * n / world)."""
    counts = np.bincount(owner, minlength=n_parts).astype(np.int64)
    csum = np.cumsum(counts)
    n = int(csum[-1]) if n_parts else 0
    ranks = np.minimum((csum - counts) * world // max(n, 1), world - 1)
    for g in range(world):
        if not (ranks == g).any():
            raise ValueError(f"rank {g} gets no part: {n_parts} parts are too few or too uneven for {world} ranks")
    return ranks.astype(np.int64)


@dataclass
class ShardPlan:
    """What one rank holds of the sharded problem (host arrays)."""
    rank: int
    world: int
    n: int                       # global DOFs
    owned: np.ndarray            # global ids of the owned DOFs, ascending
    ghost: np.ndarray            # global ids of the ghosts, by (owner rank, id)
    ghost_ptr: np.ndarray        # (world + 1,) ghosts of rank q: ghost[ghost_ptr[q]:ghost_ptr[q+1]]
    A_own: sps.csr_matrix        # owned rows, local columns (n_own x n_ext)
    A_ext: sps.csr_matrix        # owned and ghost rows and columns (blocks are cut from it)
    sub_ptr: np.ndarray          # local subdomains in local numbering
    sub_idx: np.ndarray
    first_sub: int               # global id of the first local subdomain
    halo_send: dict = field(default_factory=dict)   # q -> local ids (owned) q needs, in q's ghost order
    yl_send: dict = field(default_factory=dict)     # q -> ylocal rows for DOFs q owns, by (DOF, subdomain)
    yl_recv: dict = field(default_factory=dict)     # q -> (offset, count) in the received rows
    comb_ptr: np.ndarray = None  # owned DOF -> entries of ylocal_ext, ascending global subdomain
    comb_src: np.ndarray = None
    R0_own: sps.csr_matrix = None  # R0[:, owned]        (n_c x n_own)
    AR_own: sps.csr_matrix = None  # (R0 A)[:, owned]    (n_c x n_own)
    P_own: sps.csr_matrix = None   # R0[:, owned]^T      (n_own x n_c)

    @property
    def n_own(self) -> int:
        return len(self.owned)

    @property
    def n_ext(self) -> int:
        return len(self.owned) + len(self.ghost)

    @property
    def n_local_rows(self) -> int:
        return len(self.sub_idx)

    @property
    def n_recv_rows(self) -> int:
        return int(sum(c for _, c in self.yl_recv.values()))


def _ext_sets(A, sub_ptr, sub_idx, dof_rank, sub_rank, world):
    """Per rank: owned DOFs (ascending) and ghosts (by owner rank, then id)."""
    n = A.shape[0]
    owned, ghosts = [], []
    for g in range(world):
        own = np.nonzero(dof_rank == g)[0]
        subs = np.nonzero(sub_rank == g)[0]
        touch = np.zeros(n, dtype=bool)
        if len(own):
            rows = A[own]
            touch[rows.indices] = True
        for i in subs:
            touch[sub_idx[sub_ptr[i]:sub_ptr[i + 1]]] = True
        touch[own] = False
        gh = np.nonzero(touch)[0]
        gh = gh[np.lexsort((gh, dof_rank[gh]))]
        owned.append(own)
        ghosts.append(gh)
    return owned, ghosts


def plan_shards(A, sub_ptr, sub_idx, owner, n_parts: int, world: int, R0=None, ranks=None) -> list[ShardPlan]:
    """Plans of the given ranks (default: all) for a problem whose subdomain i
    was grown from part i of ``owner``. ``R0`` (``n_c x n``) is the coarse
    restriction, or None for a one-level method."""
    A = sps.csr_matrix(A)
    A.sort_indices()
    n = A.shape[0]
    owner = np.asarray(owner, dtype=np.int64)
    sub_ptr = np.asarray(sub_ptr, dtype=np.int64)
    sub_idx = np.asarray(sub_idx, dtype=np.int64)
    if len(sub_ptr) - 1 != n_parts:
        raise ValueError("one subdomain per part is required (subdomain i grown from part i)")
    sub_rank = part_ranks(owner, n_parts, world)
    dof_rank = sub_rank[owner]
    owned, ghosts = _ext_sets(A, sub_ptr, sub_idx, dof_rank, sub_rank, world)
    for g in range(world):
        if len(owned[g]) == 0:
            raise ValueError(f"rank {g} owns no DOF")
    # local numbering of every rank: owned, then ghosts
    l_of = []
    for g in range(world):
        m = np.full(n, -1, dtype=np.int64)
        m[owned[g]] = np.arange(len(owned[g]))
        m[ghosts[g]] = len(owned[g]) + np.arange(len(ghosts[g]))
        l_of.append(m)
    # per rank, its (global subdomain, position) entries with their DOFs
    ent_dof = sub_idx
    ent_sub = np.repeat(np.arange(n_parts), np.diff(sub_ptr))
    ent_rank = sub_rank[ent_sub]
    AR = None if R0 is None else sps.csr_matrix(R0 @ A)
    R0c = None if R0 is None else sps.csc_matrix(R0)
    plans = []
    for g in (range(world) if ranks is None else ranks):
        own, gh = owned[g], ghosts[g]
        ext = np.concatenate([own, gh])
        lg = l_of[g]
        A_ext = sps.csr_matrix(A[ext][:, ext])
        A_ext.sort_indices()
        A_own = sps.csr_matrix(A[own][:, ext])
        A_own.sort_indices()
        assert A_own.nnz == A[own].nnz, "a matrix neighbour of an owned DOF is missing from the ghosts"
        subs = np.nonzero(sub_rank == g)[0]
        first = int(subs[0]) if len(subs) else 0
        lp = sub_ptr[subs[0]:subs[-1] + 2] - sub_ptr[subs[0]] if len(subs) else np.zeros(1, np.int64)
        e0, e1 = (int(sub_ptr[subs[0]]), int(sub_ptr[subs[-1] + 1])) if len(subs) else (0, 0)
        li = lg[sub_idx[e0:e1]]
        assert (li >= 0).all()
        ghost_ptr = np.zeros(world + 1, dtype=np.int64)
        ghost_ptr[1:] = np.cumsum(np.bincount(dof_rank[gh], minlength=world))
        plan = ShardPlan(rank=g, world=world, n=n, owned=own, ghost=gh, ghost_ptr=ghost_ptr, A_own=A_own,
                         A_ext=A_ext, sub_ptr=lp.astype(np.int64), sub_idx=li.astype(np.int32), first_sub=first)
        # halo: the DOFs of mine that rank q holds as ghosts, in q's ghost order
        for q in range(world):
            if q == g:
                continue
            need = ghosts[q][dof_rank[ghosts[q]] == g]
            if len(need):
                plan.halo_send[q] = lg[need]
        # reverse exchange: my entries whose DOF another rank owns, by (DOF, subdomain)
        mine = np.arange(e0, e1)
        for q in range(world):
            if q == g:
                continue
            sel = mine[dof_rank[ent_dof[mine]] == q]
            if len(sel):
                sel = sel[np.lexsort((sel, ent_dof[sel]))]
                plan.yl_send[q] = (sel - e0).astype(np.int64)
        # received rows: from every q, its entries for my DOFs, same order
        off = 0
        recv_ent = []
        for q in range(world):
            if q == g:
                continue
            ents = np.nonzero((ent_rank == q) & (dof_rank[ent_dof] == g))[0]
            if len(ents):
                ents = ents[np.lexsort((ents, ent_dof[ents]))]
                plan.yl_recv[q] = (off, len(ents))
                recv_ent.append((ents, e1 - e0 + off))
                off += len(ents)
        # combine map over ylocal_ext = [local rows | received rows]: every
        # owned DOF's entries by global subdomain (= global entry index order)
        loc_own = np.nonzero(dof_rank[ent_dof[mine]] == g)[0]
        all_ent = [mine[loc_own]]
        all_pos = [loc_own.astype(np.int64)]
        for ents, base in recv_ent:
            all_ent.append(ents)
            all_pos.append(base + np.arange(len(ents), dtype=np.int64))
        all_ent = np.concatenate(all_ent)
        all_pos = np.concatenate(all_pos)
        d_loc = lg[ent_dof[all_ent]]
        order = np.lexsort((all_ent, d_loc))
        plan.comb_src = all_pos[order].astype(np.int32)
        plan.comb_ptr = np.zeros(len(own) + 1, dtype=np.int64)
        plan.comb_ptr[1:] = np.cumsum(np.bincount(d_loc, minlength=len(own)))
        plan.comb_ptr = plan.comb_ptr.astype(np.int32)
        if R0 is not None:
            plan.R0_own = sps.csr_matrix(R0c[:, own])
            plan.R0_own.sort_indices()
            plan.AR_own = sps.csr_matrix(sps.csc_matrix(AR)[:, own])
            plan.AR_own.sort_indices()
            plan.P_own = sps.csr_matrix(plan.R0_own.T)
            plan.P_own.sort_indices()
        plans.append(plan)
    return plans


# ---------------------------------------------------------------------------
# communicators
# ---------------------------------------------------------------------------

class DistComm:
    """One shard per process over ``torch.distributed`` (NCCL between GPUs, gloo
    on CPU): point-to-point exchanges batched per step, sums by all-reduce."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.shards = [dist.get_rank(group)]

    def allreduce(self, ts: list[torch.Tensor]) -> None:
        self.dist.all_reduce(ts[0], group=self.group)

    def exchange(self, sends: list[dict], recvs: list[dict]) -> None:
        """``sends[0][q]`` goes to rank q, ``recvs[0][q]`` is filled from rank q."""
        P2P = self.dist.P2POp
        ops = [P2P(self.dist.isend, t, q, self.group) for q, t in sorted(sends[0].items())]
        ops += [P2P(self.dist.irecv, t, q, self.group) for q, t in sorted(recvs[0].items())]
        if ops:
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()


class LocalComm:
    """All ``world`` shards in one process: an exchange is a copy, a sum adds
    the shards' tensors in rank order and writes the total to every shard."""

    def __init__(self, world: int):
        self.world = world
        self.shards = list(range(world))

    def allreduce(self, ts: list[torch.Tensor]) -> None:
        tot = ts[0].clone()
        for t in ts[1:]:
            tot += t
        for t in ts:
            t.copy_(tot)

    def exchange(self, sends: list[dict], recvs: list[dict]) -> None:
        for g, snd in enumerate(sends):
            for q, t in snd.items():
                recvs[q][g].copy_(t)


# ---------------------------------------------------------------------------
# exchanges (any device: CUDA tensors over NCCL, CPU tensors over gloo)
# ---------------------------------------------------------------------------

class ShardLinks:
    """A shard's exchange lists as index tensors on ``device``, and the views
    into its vectors that the exchanges fill."""

    def __init__(self, plan: ShardPlan, device):
        self.plan = plan
        self.rank = plan.rank
        self.n_own, self.n_ext = plan.n_own, plan.n_ext
        self.T = plan.n_local_rows
        self.n_recv = plan.n_recv_rows
        self.halo_send = {q: torch.as_tensor(v, device=device) for q, v in plan.halo_send.items()}
        self.yl_send = {q: torch.as_tensor(v, device=device) for q, v in plan.yl_send.items()}
        self.halo_from = [q for q in range(plan.world)
                          if q != plan.rank and plan.ghost_ptr[q + 1] > plan.ghost_ptr[q]]

    def buffers(self, R: int, acc_dtype, device) -> dict:
        """Send buffers: ghost rows for every neighbour (FP64) and ylocal rows."""
        return {"halo": {q: torch.zeros(len(v) * R, dtype=torch.float64, device=device)
                         for q, v in self.halo_send.items()},
                "yl": {q: torch.zeros(len(v) * R, dtype=acc_dtype, device=device) for q, v in self.yl_send.items()}}

    def ghost_view(self, vec: torch.Tensor, q: int, R: int) -> torch.Tensor:
        gp = self.plan.ghost_ptr
        return vec[(self.n_own + int(gp[q])) * R:(self.n_own + int(gp[q + 1])) * R]

    def recv_views(self, ylocal: torch.Tensor, R: int) -> dict:
        return {q: ylocal[(self.T + off) * R:(self.T + off + c) * R] for q, (off, c) in self.plan.yl_recv.items()}


def halo_exchange(comm, links: list, vecs: list, bufs: list, R: int) -> None:
    """Fill the ghost rows of every shard's ``(n_ext, R)`` vector from their owners."""
    sends, recvs = [], []
    for lk, v, b in zip(links, vecs, bufs):
        vm = v.view(lk.n_ext, R)
        snd = {}
        for q, idx in lk.halo_send.items():
            out = b["halo"][q]
            torch.index_select(vm, 0, idx, out=out.view(len(idx), R))
            snd[q] = out
        sends.append(snd)
        recvs.append({q: lk.ghost_view(v, q, R) for q in lk.halo_from})
    comm.exchange(sends, recvs)


def reverse_exchange(comm, links: list, ylocals: list, bufs: list, R: int) -> None:
    """Send the ylocal rows of other ranks' DOFs to their owners, which append
    them after their own T rows."""
    sends, recvs = [], []
    for lk, yl, b in zip(links, ylocals, bufs):
        ym = yl[: max(lk.T, 1) * R].view(-1, R)
        snd = {}
        for q, idx in lk.yl_send.items():
            out = b["yl"][q]
            torch.index_select(ym, 0, idx, out=out.view(len(idx), R))
            snd[q] = out
        sends.append(snd)
        recvs.append(lk.recv_views(yl, R))
    comm.exchange(sends, recvs)


# ---------------------------------------------------------------------------
# the sharded solver (CUDA kernels through the C ABI)
# ---------------------------------------------------------------------------

def _csr_i32(M: sps.csr_matrix, device):
    M = sps.csr_matrix(M)
    M.sort_indices()
    return (torch.as_tensor(M.indptr.astype(np.int32), device=device),
            torch.as_tensor(M.indices.astype(np.int32), device=device),
            torch.as_tensor(M.data.astype(np.float64), device=device))


def _torch_csr(M: sps.csr_matrix, device) -> torch.Tensor:
    M = sps.csr_matrix(M)
    return torch.sparse_csr_tensor(torch.as_tensor(M.indptr.astype(np.int64)),
                                   torch.as_tensor(M.indices.astype(np.int64)),
                                   torch.as_tensor(M.data.astype(np.float64)), M.shape).to(device)


class _Shard:
    """Device state of one rank: its rows of A, its local Schwarz operator (no
    coarse space), the combine map, the coarse pieces and the exchange lists."""

    def __init__(self, plan: ShardPlan, block_dtype, device, inverse=None):
        from . import solvers as S

        self.plan = plan
        self.device = device
        self.n_own, self.n_ext = plan.n_own, plan.n_ext
        self.T = plan.n_local_rows
        self.n_recv = plan.n_recv_rows
        self.A = S._SellMatrix(_torch_csr(plan.A_own, device))
        self.A.spmm_cluster = 0  # rectangular local block (ghost columns): rows in their own order
        pc = S.AdditiveSchwarz(torch.float64, S.Inv(block_dtype), None)
        pc.max_parts = 1  # one ylocal slice: rows are (subdomain, position) entries
        pc.setup(_torch_csr(plan.A_ext, device), subdomains=(plan.sub_ptr, plan.sub_idx), block_size=1)
        self.pc = pc
        self.comb_ptr = torch.as_tensor(plan.comb_ptr, device=device)
        self.comb_src = torch.as_tensor(plan.comb_src, device=device)
        self.links = ShardLinks(plan, device)
        self.n_c = 0
        if plan.R0_own is not None:
            self.n_c = plan.R0_own.shape[0]
            self.R0 = _csr_i32(plan.R0_own, device)
            self.AR = _csr_i32(plan.AR_own, device)
            P = plan.P_own
            if P.nnz == P.shape[0] and bool((np.diff(P.indptr) == 1).all()) and bool((P.data == 1.0).all()):
                self.P = (None, torch.as_tensor(P.indices.astype(np.int32), device=device), None)
            else:
                self.P = _csr_i32(P, device)
            self.inverse = inverse
        self.bufs = {}

    def work(self, R: int, maxiter: int):
        """The solve buffers for R columns (one set per R: the local operator's
        scratch ``ylocal`` is a view of this set's ``ylocal``)."""
        from . import _lib as L

        w = self.bufs.get(R)
        if w is not None:
            if w.hist.numel() < (maxiter + 1) * R:
                w.hist = torch.zeros((maxiter + 1) * R, dtype=torch.float64, device=self.device)
            return w
        f = dict(dtype=torch.float64, device=self.device)
        acc = self.pc.acc_dtype
        w = type("ShardWork", (), {})()
        w.R = R
        w.b = torch.zeros(self.n_own * R, **f)
        w.x = torch.zeros(self.n_ext * R, **f)
        w.r = torch.zeros(self.n_ext * R, **f)
        w.p = torch.zeros(self.n_ext * R, **f)
        w.z = torch.zeros(self.n_own * R, **f)
        w.q = torch.zeros(self.n_own * R, **f)
        w.y = torch.zeros(self.n_own * R, **f)
        w.st = torch.zeros(L.ST_COUNT * R, **f)
        w.ist = torch.zeros(L.IST_COUNT * R + L.G_COUNT, dtype=torch.int32, device=self.device)
        w.hist = torch.zeros((maxiter + 1) * R, **f)
        w.partials = torch.zeros(int(L.lib().ddx_partials_len(R)), **f)
        w.tickets = torch.zeros(L.TICKETS, dtype=torch.int32, device=self.device)
        w.ylocal = torch.zeros(max(self.T + self.n_recv, 1) * R, dtype=acc, device=self.device)
        s = self.pc.scratch(R)
        s["ylocal"] = w.ylocal[: max(self.T, 1) * R]  # the local apply writes the first T rows in place
        if self.n_c:
            w.w = torch.zeros(self.n_c * R, **f)
            w.yc = torch.zeros(self.n_c * R, **f)
        w.send = self.links.buffers(R, acc, self.device)
        self.bufs[R] = w
        return w


class ShardedCG:
    """Two-level Schwarz PCG with the subdomains split over ranks.

    ``method`` is ``"additive"`` or ``"hybrid"``; ``block_dtype`` the storage of
    the local inverse blocks (FP64 / FP32 / BF16 / FP16, per-block scaled);
    ``flexible`` defaults to on below FP64 blocks, as ``CG`` does. ``setup``
    takes the global problem on the host (every rank builds its own plan from
    it); ``solve`` takes the global right-hand side (every rank passes the
    same) and returns the global solution on every rank, with the reference's
    metadata (``iterations``, ``residual norms``).
    """

    def __init__(self, method: str = "hybrid", block_dtype=torch.float64, rtol: float = 1e-7, atol: float = 0.0,
                 maxiter: int = 1000, flexible: bool | None = None, check_every: int = 8):
        assert method in ("additive", "hybrid")
        self.method = method
        self.block_dtype = block_dtype
        self.rtol, self.atol, self.maxiter = rtol, atol, maxiter
        self.flexible = (block_dtype != torch.float64) if flexible is None else flexible
        self.check_every = check_every

    def setup(self, A, sub_ptr, sub_idx, owner, n_parts: int, R0=None, comm=None, device=None) -> None:
        from . import cudss

        self.comm = comm if comm is not None else LocalComm(1)
        self.world = self.comm.world
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        A = sps.csr_matrix(A)
        self.n = A.shape[0]
        plans = plan_shards(A, sub_ptr, sub_idx, owner, n_parts, self.world, R0, ranks=self.comm.shards)
        inverse = None
        if R0 is not None:
            Ac = sps.csr_matrix(R0 @ A @ R0.T)
            inverse = cudss._dense_inverse(torch.as_tensor(Ac.toarray(), device=dev))
        self.shards = [_Shard(p, self.block_dtype, dev, inverse) for p in plans]
        self.n_c = self.shards[0].n_c

    # -- exchanges ---------------------------------------------------------
    def _halo(self, name: str, R: int) -> None:
        """Ghost rows of vector ``name`` from their owners."""
        ws = [sh.bufs[self._key] for sh in self.shards]
        halo_exchange(self.comm, [sh.links for sh in self.shards], [getattr(w, name) for w in ws],
                      [w.send for w in ws], R)

    def _reverse(self, R: int) -> None:
        """ylocal rows of other ranks' DOFs to their owners."""
        ws = [sh.bufs[self._key] for sh in self.shards]
        reverse_exchange(self.comm, [sh.links for sh in self.shards], [w.ylocal for w in ws],
                         [w.send for w in ws], R)

    def _sum_totals(self, kind: int, R: int) -> None:
        """Sum the parked totals over the ranks, then the epilogue on every shard."""
        from . import _lib as L

        ws = [sh.bufs[self._key] for sh in self.shards]
        self.comm.allreduce([w.st[L.ST_T0 * R:(L.ST_T1 + 1) * R] for w in ws])
        for w in ws:
            L.call("ddx_pcg_finalize", R, kind, L.ptr(w.st), L.ptr(w.ist), L.ptr(w.hist), L.stream_ptr())

    def _coarse_from(self, src: str, mat: str, R: int) -> None:
        """yc = A_C^-1 sum_ranks mat[:, own] src_own (one all-reduce of n_c x R)."""
        for sh in self.shards:
            w = sh.bufs[self._key]
            sh.pc._restrict(*getattr(sh, mat), getattr(w, src), w.w, R)
        self.comm.allreduce([sh.bufs[self._key].w for sh in self.shards])
        from . import _lib as L

        for sh in self.shards:
            w = sh.bufs[self._key]
            L.call("ddx_coarse_gemv_f64", self.n_c, R, L.ptr(sh.inverse), L.ptr(w.w), L.ptr(w.yc), L.ptr(w.ist),
                   L.stream_ptr())

    def _combine(self, sh, w, R, out, ylocal=True, u=None, prolong=False, sign=1.0, dots=False) -> None:
        from . import _lib as L

        p_ptr = p_col = p_val = yc = None
        if prolong:
            p_ptr, p_col, p_val = sh.P
            yc = w.yc
        dp, ds, yl = (sh.comb_ptr, sh.comb_src, w.ylocal) if ylocal else (None, None, None)
        L.call("ddx_schwarz_combine", sh.n_own, R, L.ptr(dp), L.ptr(ds), L.ptr(yl), L.DTYPE_CODE[sh.pc.acc_dtype],
               L.ptr(u), L.ptr(p_ptr), L.ptr(p_col), L.ptr(p_val), L.ptr(yc), float(sign), L.ptr(out), int(dots),
               L.ptr(w.r) if dots else None, L.ptr(w.q) if dots else None,
               L.ptr(w.st) if dots else None, L.ptr(w.ist) if dots else None,
               L.ptr(w.partials) if dots else None, L.ptr(w.tickets) if dots else None, L.stream_ptr())

    # -- PCG steps -----------------------------------------------------------
    def _precondition(self, R: int) -> None:
        """z = M r (owned rows) with r.z (and z.q) summed over the ranks -> beta."""
        from . import _lib as L

        self._halo("r", R)
        hybrid = self.method == "hybrid" and self.n_c
        if self.method == "additive" and self.n_c:
            self._coarse_from("r", "R0", R)
        for sh in self.shards:
            w = sh.bufs[self._key]
            sh.pc._local(w.r, R, w.ist, w.st)
        self._reverse(R)
        if hybrid:
            for sh in self.shards:
                w = sh.bufs[self._key]
                self._combine(sh, w, R, w.y)
            self._coarse_from("y", "AR", R)
            for sh in self.shards:
                w = sh.bufs[self._key]
                self._combine(sh, w, R, w.z, ylocal=False, u=w.y, prolong=True, sign=-1.0, dots=True)
        else:
            for sh in self.shards:
                w = sh.bufs[self._key]
                self._combine(sh, w, R, w.z, prolong=bool(self.n_c), sign=1.0, dots=True)
        self._sum_totals(L.FIN_RZ, R)

    def _iteration(self, R: int) -> None:
        from . import _lib as L

        self._precondition(R)
        for sh in self.shards:
            w = sh.bufs[self._key]
            L.call("ddx_pcg_update_p", sh.n_own, R, L.ptr(w.z), L.ptr(w.p), L.ptr(w.st), L.ptr(w.ist),
                   L.stream_ptr())
        self._halo("p", R)
        for sh in self.shards:
            w = sh.bufs[self._key]
            sh.A.launch(w.p, w.q, R, L.SPMV_PQ, w)
        self._sum_totals(L.FIN_PQ, R)
        for sh in self.shards:
            w = sh.bufs[self._key]
            L.call("ddx_pcg_update_xr", sh.n_own, R, L.ptr(w.x), L.ptr(w.r), L.ptr(w.p), L.ptr(w.q), L.ptr(w.st),
                   L.ptr(w.ist), L.ptr(w.hist), L.ptr(w.partials), L.ptr(w.tickets), L.stream_ptr())
        self._sum_totals(L.FIN_RR, R)

    def solve(self, rhs: torch.Tensor):
        """Solve ``A x = rhs`` (global ``(n,)`` or ``(n, R)``, the same on every
        rank); returns the global x on every rank and the metadata."""
        from . import _lib as L
        from .solvers import ConvergenceNotAchieved

        n = self.n
        R = 1 if rhs.dim() == 1 else rhs.shape[1]
        Rp = 1 << max(0, (R - 1).bit_length())
        if Rp > 64:
            raise ValueError("at most 64 right-hand sides per solve")
        maxiter = self.maxiter or n * 10
        self._key = Rp
        B = torch.zeros((n, Rp), dtype=torch.float64, device=self.device)
        B[:, :R] = rhs.reshape(n, R).to(self.device, torch.float64)
        for sh in self.shards:
            w = sh.work(Rp, maxiter)
            own = torch.as_tensor(sh.plan.owned, device=self.device)
            w.b.view(sh.n_own, Rp).copy_(B[own])
            for t in (w.x, w.r, w.p, w.z, w.q, w.y):
                t.zero_()
            L.call("ddx_pcg_reset", Rp, L.ptr(w.st), L.ptr(w.ist), maxiter, int(self.flexible), float(self.rtol),
                   float(self.atol), L.stream_ptr())
            w.ist[L.IST_COUNT * Rp + L.G_DEFER] = 1
        if self.method == "hybrid" and self.n_c:
            # x0 = R0^T A_C^-1 R0 b
            self._coarse_from("b", "R0", Rp)
            for sh in self.shards:
                w = sh.bufs[self._key]
                self._combine(sh, w, Rp, w.x, ylocal=False, u=w.x, prolong=True, sign=1.0)
        self._halo("x", Rp)
        for sh in self.shards:
            w = sh.bufs[self._key]
            sh.A.launch(w.x, w.r, Rp, L.SPMV_RES_INIT, w, b=w.b)
        self._sum_totals(L.FIN_INIT, Rp)
        w0 = self.shards[0].bufs[self._key]
        done = 0
        k = max(1, int(self.check_every))
        active = int(w0.ist[L.IST_COUNT * Rp + L.G_NACTIVE].item())
        while active > 0 and done < maxiter:
            for _ in range(min(k, maxiter - done)):
                self._iteration(Rp)
            done += min(k, maxiter - done)
            active = int(w0.ist[L.IST_COUNT * Rp + L.G_NACTIVE].item())
        # the global solution on every rank: owned rows scattered, summed over ranks
        X = torch.zeros((n, Rp), dtype=torch.float64, device=self.device)
        parts = []
        for sh in self.shards:
            w = sh.bufs[self._key]
            Xg = X if len(self.shards) == 1 else torch.zeros_like(X)
            Xg[torch.as_tensor(sh.plan.owned, device=self.device)] = w.x[: sh.n_own * Rp].view(sh.n_own, Rp)
            parts.append(Xg)
        self.comm.allreduce(parts)
        X = parts[0]
        ist = w0.ist[: L.IST_COUNT * Rp].view(L.IST_COUNT, Rp).cpu()
        st = w0.st.view(L.ST_COUNT, Rp).cpu()
        hist = w0.hist.view(-1, Rp)[: maxiter + 1].cpu()
        its, norms, failed = [], [], False
        for j in range(R):
            it = int(ist[L.IST_ITERS, j])
            conv = float(hist[it, j]) < float(st[L.ST_ATOL, j]) or (float(st[L.ST_BB, j]) == 0.0 and it == 0)
            if conv:
                its.append(it)
                norms.append([float(v) for v in hist[: it + 1, j]])
                failed |= it + 1 >= maxiter
            else:
                its.append(maxiter - 1)
                norms.append([float(v) for v in hist[:maxiter, j]])
                failed = True
        meta = ({"iterations": its[0], "residual norms": norms[0]} if rhs.dim() == 1 else
                {"iterations": its, "residual norms": norms})
        x = X[:, :R].reshape(rhs.shape).to(rhs.dtype)
        if failed:
            raise ConvergenceNotAchieved(meta)
        return x, meta
