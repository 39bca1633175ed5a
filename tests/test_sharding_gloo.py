"""The domain-sharded path's host side on CPU: plans, and the product's exchange
code (``halo_exchange``, ``reverse_exchange``, ``DistComm``) run by world_size
2 and 3 gloo ranks, each doing its local arithmetic in NumPy/torch on the CPU.

The distributed PCG below is the sharded solver's step order (halo of r, local
products, reverse exchange, combine in global subdomain order, coarse
all-reduce, all-reduced dots) with the oracle's blocks; it must reproduce the
oracle's one-process solve.
"""
import os
import socket
import traceback

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from helpers import p1_case, q1_case


def _case(name):
    if name == "q1_2d_p0":
        return q1_case(2, 24, 4)
    if name == "q1_3d_q1coarse":
        return q1_case(3, 12, 3, kappa_seed=4, coarse="q1")
    return p1_case(30, 8)


@pytest.mark.parametrize("case", ["q1_2d_p0", "q1_3d_q1coarse", "p1_rcb"])
@pytest.mark.parametrize("world", [2, 3, 4])
def test_plan_invariants(case, world):
    from dd_solvers_b200.sharding import plan_shards

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = _case(case)
    n = A.shape[0]
    plans = plan_shards(A, sub_ptr, sub_idx, owner, nparts, world, R0)
    # owned sets partition the DOFs; subdomains are split in contiguous runs
    assert np.array_equal(np.sort(np.concatenate([p.owned for p in plans])), np.arange(n))
    assert [p.first_sub for p in plans] == sorted(p.first_sub for p in plans)
    assert sum(len(p.sub_ptr) - 1 for p in plans) == nparts
    x = np.random.default_rng(1).standard_normal(n)
    for p in plans:
        ext = np.concatenate([p.owned, p.ghost])
        # local rows of A reproduce the global rows
        assert np.allclose(p.A_own @ x[ext], (A @ x)[p.owned], rtol=0, atol=1e-12)
        # every ghost slice of a neighbour is what that neighbour sends
        for q, idx in p.halo_send.items():
            g = plans[q]
            assert np.array_equal(p.owned[idx], g.ghost[g.ghost_ptr[p.rank]:g.ghost_ptr[p.rank + 1]])
        # the combine lists every subdomain holding an owned DOF exactly once
        counts = np.bincount(sub_idx, minlength=n)[p.owned]
        assert np.array_equal(np.diff(p.comb_ptr), counts)
        # reverse exchange sizes agree on both sides
        for q, (off, c) in p.yl_recv.items():
            assert len(plans[q].yl_send[p.rank]) == c
        # the owned columns of the coarse products sum to the global ones
    w = sum(p.R0_own @ x[p.owned] for p in plans)
    assert np.allclose(w, R0 @ x, rtol=0, atol=1e-12)
    w = sum(p.AR_own @ x[p.owned] for p in plans)
    assert np.allclose(w, (R0 @ A) @ x, rtol=0, atol=1e-11)


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _sharded_pcg(case, method, rank, world, rtol):
    """One rank of the sharded PCG with NumPy/torch CPU arithmetic and the
    product's plan and exchanges."""
    import scipy.linalg as sla

    from dd_solvers_b200.sharding import DistComm, ShardLinks, halo_exchange, plan_shards, reverse_exchange
    from oracle import restatement as orc

    P, A, owner, nparts, sub_ptr, sub_idx, R0 = _case(case)
    n = A.shape[0]
    M = orc.Schwarz(A, sub_ptr, sub_idx, R0)
    b = np.random.default_rng(11).uniform(-1, 1, n)
    comm = DistComm()
    (plan,) = plan_shards(A, sub_ptr, sub_idx, owner, nparts, world, R0, ranks=[rank])
    lk = ShardLinks(plan, "cpu")
    bufs = lk.buffers(1, torch.float64, "cpu")
    n_own, n_ext = plan.n_own, plan.n_ext

    def allsum(v):
        t = torch.as_tensor(np.atleast_1d(np.asarray(v, dtype=np.float64))).clone()
        comm.allreduce([t])
        return t.numpy()

    def halo(v):
        t = torch.as_tensor(v)
        halo_exchange(comm, [lk], [t], [bufs], 1)
        return t.numpy()

    def coarse(mat, v_own):
        return sla.cho_solve(M.Ac_cho, allsum(mat @ v_own))

    def apply(r_ext):
        r_ext = halo(r_ext)
        yl = np.zeros(lk.T + lk.n_recv)
        pos = 0
        for i in range(len(plan.sub_ptr) - 1):
            idx = plan.sub_idx[plan.sub_ptr[i]:plan.sub_ptr[i + 1]]
            g = plan.first_sub + i
            yl[pos:pos + len(idx)] = M.scales[g] * (M.blocks[g] @ r_ext[idx])
            pos += len(idx)
        ylt = torch.as_tensor(yl)
        reverse_exchange(comm, [lk], [ylt], [bufs], 1)
        yl = ylt.numpy()
        y = np.array([yl[plan.comb_src[plan.comb_ptr[d]:plan.comb_ptr[d + 1]]].sum() for d in range(n_own)])
        if method == "hybrid":
            return y - plan.P_own @ coarse(plan.AR_own, y)
        return y + plan.P_own @ coarse(plan.R0_own, r_ext[:n_own])

    b_own = b[plan.owned]
    atol = rtol * float(np.sqrt(allsum(b_own @ b_own)[0]))
    x = np.zeros(n_ext)
    if method == "hybrid":
        x[:n_own] = plan.P_own @ coarse(plan.R0_own, b_own)
    x = halo(x)
    r = np.zeros(n_ext)
    r[:n_own] = b_own - plan.A_own @ x
    p = np.zeros(n_ext)
    rho_prev = None
    its = 0
    for it in range(2000):
        rn = float(np.sqrt(allsum(r[:n_own] @ r[:n_own])[0]))
        if rn < atol:
            break
        z = apply(r.copy())
        rho = float(allsum(r[:n_own] @ z)[0])
        p[:n_own] = z if rho_prev is None else z + (rho / rho_prev) * p[:n_own]
        p = halo(p)
        q = plan.A_own @ p
        alpha = rho / float(allsum(p[:n_own] @ q)[0])
        x[:n_own] += alpha * p[:n_own]
        r[:n_own] -= alpha * q
        rho_prev = rho
        its = it + 1
    X = np.zeros(n)
    X[plan.owned] = x[:n_own]
    return allsum(X), its


def _worker(rank, world, port, case, method, q):
    import datetime

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        X, its = _sharded_pcg(case, method, rank, world, 1e-10)
        q.put((rank, X, its))
        dist.destroy_process_group()
    except Exception:
        q.put((rank, "exception: " + traceback.format_exc(), 0))


def _run(case, method, world, timeout=240):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, method, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=timeout) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        if p.is_alive():
            p.kill()
    return sorted(out, key=lambda t: t[0])


@pytest.mark.parametrize("case,method,world", [("q1_2d_p0", "hybrid", 2), ("q1_3d_q1coarse", "hybrid", 3),
                                               ("p1_rcb", "additive", 2), ("q1_3d_q1coarse", "additive", 2)])
def test_sharded_pcg_over_gloo_matches_oracle(case, method, world):
    from oracle import restatement as orc

    res = _run(case, method, world)
    for rank, X, its in res:
        assert not isinstance(X, str), X
    P, A, owner, nparts, sub_ptr, sub_idx, R0 = _case(case)
    b = np.random.default_rng(11).uniform(-1, 1, A.shape[0])
    M = orc.Schwarz(A, sub_ptr, sub_idx, R0)
    if method == "hybrid":
        xr, om = orc.pcg(A, b, M.hybrid, rtol=1e-10, T0=M.T0)
    else:
        xr, om = orc.pcg(A, b, M.additive, rtol=1e-10)
    for rank, X, its in res:
        assert abs(its - om["iterations"]) <= 1, (its, om["iterations"])
        assert np.linalg.norm(X - xr) <= 1e-10 * np.linalg.norm(xr)
    # every rank holds the same solution
    assert all(np.array_equal(res[0][1], X) for _, X, _ in res)
