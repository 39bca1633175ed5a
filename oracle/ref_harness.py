"""ORACLE (test infrastructure only): run the reference's own solver code on CPU.

This loads ``src/dd_solvers/dd_solvers/solvers.py`` from a checkout of the
reference named by the environment variable ``DDX_REFERENCE_ROOT`` (required;
the checkout is a development-time input, not part of this package) and runs
its ``CG``, ``AdditiveSchwarz``,
``HybridSchwarz``, ``Inv``, ``asm_permutation``, ``permute_csr_tensor`` and
``inverse_permutation`` verbatim on CPU tensors. Only the pieces that need a
GPU or an absent library are replaced by same-math CPU equivalents:

* ``pyamgx``                       -> stub with a no-op ``initialize``;
* ``gemv_strided_batched``         -> ``(M.to(v.dtype) @ v[..., None])[..., 0]``
                                      (same upcast-then-accumulate-in-vector-dtype rule,
                                      ``cpp/gemv_kernels.cu:45-54``);
* ``cudss.spd_factorize``          -> dense FP64 Cholesky (``scipy.linalg.cho_factor``);
* ``sort_csr`` / ``gather_csr``    -> SciPy ``sort_indices`` / ``sum_duplicates``;
* ``CUDSS.setup/solve``            -> same calls minus the ``is_cuda`` asserts;
* numba setup kernels              -> run under the numba CUDA simulator for small
                                      matrices, or by the vectorised NumPy restatement
                                      of the same loops (``solvers.py:407-481``) at scale;
* ``torch.linalg.inv``             -> ``numpy.linalg.inv`` (MKL trips on large CPU batches);
* ``torch.compile``                -> disabled (``TORCHDYNAMO_DISABLE=1``).

Used by ``tests/golden/make_golden.py`` to write the committed fixtures.
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types

REF_ROOT = os.environ.get("DDX_REFERENCE_ROOT")
_SIM_MAX_ROWS = 2000


def load(ref_root: str | None = REF_ROOT):
    if not ref_root:
        raise RuntimeError("set DDX_REFERENCE_ROOT to a checkout of the reference (mgr0dzicki/dd-solvers)")
    os.environ.setdefault("TORCHDYNAMO_DISABLE", "1")
    os.environ.setdefault("NUMBA_ENABLE_CUDASIM", "1")
    import numpy as np
    import scipy.linalg as sla
    import scipy.sparse as sps
    import torch

    src = os.path.join(ref_root, "src", "dd_solvers", "dd_solvers", "solvers.py")
    if not os.path.exists(src):
        raise FileNotFoundError(src)

    pkg = types.ModuleType("ddref")
    pkg.__path__ = []
    sys.modules["ddref"] = pkg
    sys.modules.setdefault("pyamgx", types.SimpleNamespace(initialize=lambda: None))

    def _csr_parts(m):
        return (m.crow_indices().numpy(), m.col_indices().numpy(), m.values().numpy(), tuple(m.shape))

    def sort_csr(matrix, num_parts=None):
        crow, col, val, shape = _csr_parts(matrix)
        s = sps.csr_matrix((val.copy(), col.astype(np.int64), crow.astype(np.int64)), shape=shape)
        s.has_sorted_indices = False
        s.sort_indices()
        return torch.sparse_csr_tensor(torch.as_tensor(s.indptr.astype(np.int32)),
                                       torch.as_tensor(s.indices.astype(np.int32)),
                                       torch.as_tensor(s.data), size=shape)

    def gather_csr(matrix):
        crow, col, val, shape = _csr_parts(matrix)
        s = sps.csr_matrix((val.copy(), col.astype(np.int64), crow.astype(np.int64)), shape=shape)
        s.sum_duplicates()
        return torch.sparse_csr_tensor(torch.as_tensor(s.indptr.astype(crow.dtype)),
                                       torch.as_tensor(s.indices.astype(col.dtype)),
                                       torch.as_tensor(s.data), size=shape)

    def csr_to_bsr(matrix, block_size):
        raise RuntimeError("FastBSR needs a GPU; use CG(bsr_matmul=False) in the harness")

    cus = types.ModuleType("ddref.cusparse")
    cus.sort_csr, cus.gather_csr, cus.csr_to_bsr = sort_csr, gather_csr, csr_to_bsr
    bsr = types.ModuleType("ddref.bsr")
    bsr.FastBSR = None
    gem = types.ModuleType("ddref.gemv")
    gem.gemv_strided_batched = lambda mat, vec, use_shared_memory=None: (mat.to(vec.dtype) @ vec[..., None])[..., 0]

    class _DenseCholesky:
        def __init__(self, A):
            self.dtype = A.dtype
            dense = A.to_dense().to(torch.float64).numpy()
            self.cf = sla.cho_factor(dense)

        def solve(self, rhs):
            return torch.as_tensor(sla.cho_solve(self.cf, rhs.to(torch.float64).numpy())).to(rhs.dtype)

    cud = types.ModuleType("ddref.cudss")
    cud.spd_factorize = _DenseCholesky
    for name, mod in (("cusparse", cus), ("bsr", bsr), ("gemv", gem), ("cudss", cud)):
        sys.modules[f"ddref.{name}"] = mod
        setattr(pkg, name, mod)

    spec = importlib.util.spec_from_file_location("ddref.solvers", src)
    solvers = importlib.util.module_from_spec(spec)
    sys.modules["ddref.solvers"] = solvers
    spec.loader.exec_module(solvers)

    # CUDSS without the is_cuda asserts (solvers.py:89-113)
    def cudss_setup(self, matrix, *args, **kwargs):
        self.solver = cud.spd_factorize(matrix)
        self.dtype = matrix.dtype

    def cudss_solve(self, rhs):
        return self.solver.solve(rhs), {}

    solvers.CUDSS.setup = cudss_setup
    solvers.CUDSS.solve = cudss_solve

    _np_inv = lambda a: torch.as_tensor(np.linalg.inv(a.numpy()))
    torch.linalg.inv = _np_inv

    # numba setup kernels: simulator when small, NumPy restatement when large
    sim_dense = solvers.construct_local_solvers_matrices_dense_kernel
    sim_count = solvers.construct_coarse_solver_matrix_count_kernel
    sim_coo = solvers.construct_coarse_solver_matrix_coo_kernel

    def _np(a):
        return a.numpy() if isinstance(a, torch.Tensor) else a

    class _Launcher:
        def __init__(self, sim, vec, crow_arg):
            self.sim, self.vec, self.crow_arg = sim, vec, crow_arg

        def __getitem__(self, cfg):
            def run(*args):
                args = [_np(a) for a in args]
                nrows = len(args[self.crow_arg]) - 1
                if nrows <= _SIM_MAX_ROWS:
                    self.sim[cfg](*args)
                else:
                    self.vec(*args)
            return run

    def _dense_np(k, crow, col, val, out):
        n = len(crow) - 1
        rows = np.repeat(np.arange(n), np.diff(crow))
        same = (col // k) == (rows // k)
        r, c = rows[same], col[same]
        out[r // k, r % k, c % k] = val[same]

    def _count_np(k, s2c, crow, col, out):
        n = len(crow) - 1
        rows = np.repeat(np.arange(n), np.diff(crow))
        blk = s2c[col // k]
        first = np.ones(len(col), dtype=bool)
        first[1:] = (blk[1:] != blk[:-1]) | (rows[1:] != rows[:-1])
        out[:] = np.bincount(rows[first], minlength=n)

    def _coo_np(k, s2c, crow, col, val, scan, out_idx, out_val):
        n = len(crow) - 1
        rows = np.repeat(np.arange(n), np.diff(crow))
        blk = s2c[col // k]
        first = np.ones(len(col), dtype=bool)
        first[1:] = (blk[1:] != blk[:-1]) | (rows[1:] != rows[:-1])
        seg = np.cumsum(first) - 1
        sums = np.zeros(int(first.sum()))
        for_each = val
        # sequential per-row accumulation order as in the kernel
        np.add.at(sums, seg, for_each)
        out_idx[0, :] = s2c[rows[first] // k]
        out_idx[1, :] = blk[first]
        out_val[:] = sums

    solvers.construct_local_solvers_matrices_dense_kernel = _Launcher(sim_dense, _dense_np, 1)
    solvers.construct_coarse_solver_matrix_count_kernel = _Launcher(sim_count, _count_np, 2)
    solvers.construct_coarse_solver_matrix_coo_kernel = _Launcher(sim_coo, _coo_np, 2)
    return solvers
