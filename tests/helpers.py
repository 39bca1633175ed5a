"""Shared problem builders for the tests (small sizes)."""
import numpy as np
import scipy.sparse as sps
import torch

from dd_solvers_b200 import partition, problems


def torch_csr(A: sps.csr_matrix, device) -> torch.Tensor:
    A = sps.csr_matrix(A)
    return torch.sparse_csr_tensor(torch.as_tensor(A.indptr.astype(np.int64)),
                                   torch.as_tensor(A.indices.astype(np.int64)),
                                   torch.as_tensor(A.data), A.shape).to(device)


def q1_case(dim=2, n_el=32, parts=4, overlap=1, kappa_seed=None, coarse="p0"):
    kappa = None
    if kappa_seed is not None:
        rng = np.random.default_rng(kappa_seed)
        kappa = np.exp(rng.standard_normal((n_el,) * dim))
    P = problems.q1_grid(dim, n_el, kappa)
    A = P.matrix
    owner, nparts = partition.box_owner(P.interior_shape, parts)
    sub_ptr, sub_idx = partition.overlapping_subdomains(A, owner, nparts, overlap)
    if coarse == "p0":
        R0 = partition.p0_restriction(owner, nparts)
    elif coarse == "q1":
        R0 = partition.q1_coarse_restriction(dim, n_el, parts)
    else:
        R0 = None
    return P, A, owner, nparts, sub_ptr, sub_idx, R0


def p1_case(n_nodes=34, parts=8, overlap=1, seed=3):
    P = problems.p1_jittered(n_nodes, 0.3, 1.0, seed)
    A = P.matrix
    owner = partition.rcb_owner(P.coords, parts)
    sub_ptr, sub_idx = partition.overlapping_subdomains(A, owner, parts, overlap)
    R0 = partition.p0_restriction(owner, parts)
    return P, A, owner, parts, sub_ptr, sub_idx, R0
