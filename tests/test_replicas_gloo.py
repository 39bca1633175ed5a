"""The N > 1 replica path on CPU: world_size 2 over gloo.

* RHS split + gather reproduces the single-process block solve (oracle PCG per rank),
* max-over-ranks timing reduction,
* a rank that fails before the collective is detected by the others through a
  short process-group timeout (host-side failure detection; no GPU involved).
"""
import os
import socket
import traceback

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, mode, q):
    import datetime

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
        from dd_solvers_b200 import partition, problems, replicas
        from oracle import restatement as orc

        if mode == "solve":
            P = problems.q1_grid(2, 16)
            A = P.matrix
            owner, nparts = partition.box_owner(P.interior_shape, 4)
            sub_ptr, sub_idx = partition.overlapping_subdomains(A, owner, nparts, 1)
            M = orc.Schwarz(A, sub_ptr, sub_idx, partition.p0_restriction(owner, nparts))
            total = 5
            B = np.random.default_rng(0).standard_normal((A.shape[0], total))
            a, b = replicas.rhs_range(total, rank, world)
            X, _ = orc.pcg_multi(A, B[:, a:b], M.hybrid, T0=M.T0, rtol=1e-10)
            full = replicas.gather_columns(torch.as_tensor(X), total)
            t = replicas.max_over_ranks(1.0 + rank)
            q.put((rank, full.numpy(), t))
        elif mode == "fail":
            if rank == 1:
                raise RuntimeError("injected failure on rank 1 before the collective")
            try:
                replicas.max_over_ranks(3.0)
                q.put((rank, "no error"))
            except Exception as e:  # the peer never joins: the collective times out
                q.put((rank, "detected: " + type(e).__name__))
        dist.destroy_process_group()
    except Exception:
        q.put((rank, "exception: " + traceback.format_exc().splitlines()[-1]))


def _run(mode, world=2, timeout=120):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=timeout) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        if p.is_alive():
            p.kill()
    return sorted(out, key=lambda t: t[0])


def test_rhs_range_partition():
    from dd_solvers_b200 import replicas

    for total in (1, 5, 16, 64):
        for world in (1, 2, 3, 8):
            spans = [replicas.rhs_range(total, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == total
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def test_replicas_solve_and_max_timing_gloo():
    from dd_solvers_b200 import partition, problems
    from oracle import restatement as orc

    res = _run("solve")
    P = problems.q1_grid(2, 16)
    A = P.matrix
    owner, nparts = partition.box_owner(P.interior_shape, 4)
    sub_ptr, sub_idx = partition.overlapping_subdomains(A, owner, nparts, 1)
    M = orc.Schwarz(A, sub_ptr, sub_idx, partition.p0_restriction(owner, nparts))
    B = np.random.default_rng(0).standard_normal((A.shape[0], 5))
    X, _ = orc.pcg_multi(A, B, M.hybrid, T0=M.T0, rtol=1e-10)
    for rank, full, t in res:
        assert np.array_equal(full, X)
        assert t == 2.0


def test_rank_failure_detected_by_timeout():
    res = _run("fail")
    assert res[1][1].startswith("exception") and "injected failure" in res[1][1]
    assert res[0][1].startswith("detected") or res[0][1].startswith("exception"), res[0][1]
