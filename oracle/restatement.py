"""ORACLE (test infrastructure only): FP64 CPU restatement of Schwarz-PCG.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module, and only as the checker or the timed CPU
baseline. The product path (``dd_solvers_b200``) never imports it.

It restates the reference's algorithm with NumPy/SciPy in FP64 and generalises
it to the cases the reference cannot express (overlapping and uneven
subdomains, a general coarse restriction, several right-hand sides,
low-precision block storage with per-block power-of-two scales):

* ``pcg``                 - ``CG.solve`` (``src/dd_solvers/dd_solvers/solvers.py:228-297``):
                            stop on ``||r|| < max(atol, rtol ||b||)`` checked at the top of
                            each iteration, Fletcher-Reeves beta, ``iterations =
                            len(residual_norms) - 1`` (276), ``ConvergenceNotAchieved``
                            when the loop index reaches ``maxiter - 1`` (294-295).
                            ``flexible=True`` swaps in the Polak-Ribiere beta.
* ``Schwarz.local``       - ``sum_i R_i^T A_i^{-1} R_i r`` (``Inv.solve``, 355-359, on the
                            ``reshape(n_solvers, -1)`` blocks of 814/878, generalised to
                            index sets).
                            ``batched=True``: the blocks of each size stacked and applied
                            by one ``torch.bmm`` (as ``Inv.solve`` batches them), with
                            ``HostCSR`` (torch's threaded CSR product, as ``CG.solve``'s
                            ``self.matrix @ p``, 264) for the sparse products: the mode the
                            timed CPU baseline runs, same results up to summation order.
* ``Schwarz.additive``    - ``AdditiveSchwarz.solve`` (811-826).
* ``Schwarz.hybrid``      - ``HybridSchwarz.solve`` (874-888): ``y - R0^T A_C^{-1} (R0 A) y``.
* ``Schwarz.T0``          - ``HybridSchwarz.T0`` (861-872).
* ``coarse_matrix``       - ``R0 A R0^T`` (``_construct_coarse_solver_matrix``, 721-771).
* ``quantize``            - ``Inv.setup`` downcast (350-353) plus the per-block
                            power-of-two scale of this package's low-precision storage.
* ``ContiguousSchwarz``   - the reference's own data layout (``SchwarzOperator.setup``,
                            571-640): equal contiguous subdomains of ``dofs_per_solver``
                            DOFs, contiguous runs of ``solvers_per_coarse`` solvers per P0
                            coarse aggregate; batched local inverses; the coarse matrix
                            ``R0 A R0^T`` factored by a sparse LU (SciPy SuperLU) where the
                            reference uses cuDSS (85-113).
"""
from __future__ import annotations

import warnings

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sps
import scipy.sparse.linalg as spla


class ConvergenceNotAchieved(Exception):
    def __init__(self, metadata):
        self.metadata = metadata
        super().__init__(f"Convergence not achieved in {metadata.get('iterations')} iterations.")


# ---------------------------------------------------------------------------
# Low-precision emulation
# ---------------------------------------------------------------------------

def round_to_bf16(x: np.ndarray) -> np.ndarray:
    """FP64 -> FP32 (nearest even) -> BF16 (nearest even), returned as FP64.

    Matches ``tensor.to(torch.float32).to(torch.bfloat16)`` for finite values.
    """
    f = np.asarray(x, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    rounding = ((b >> 16) & 1) + 0x7FFF
    b = ((b + rounding) & 0xFFFF0000).astype(np.uint32)
    return b.view(np.float32).astype(np.float64)


def round_to(x: np.ndarray, dtype: str) -> np.ndarray:
    if dtype == "f64":
        return np.asarray(x, dtype=np.float64)
    if dtype == "f32":
        return np.asarray(x, dtype=np.float32).astype(np.float64)
    if dtype == "f16":
        return np.asarray(x, dtype=np.float32).astype(np.float16).astype(np.float64)
    if dtype == "bf16":
        return round_to_bf16(x)
    raise ValueError(dtype)


def rhs_scale(norm: float, dtype: str) -> float:
    """Per-RHS power-of-two scale of the 16-bit residual pack: ``norm * s`` in
    ``[2**(top-1), 2**top)``, top 14 for FP16 and 0 for BF16 (1 for a zero or
    non-finite norm)."""
    if not (norm > 0.0) or not np.isfinite(norm):
        return 1.0
    e = int(np.frexp(norm)[1])
    e = max(-100, min(100, e))
    return float(2.0 ** ((14 if dtype == "f16" else 0) - e))


def rhs_terms(r: np.ndarray, dtype: str, terms: int, scaled: bool = False) -> np.ndarray:
    """The residual a tensor-core apply multiplies: ``sum_t h_t / s_j`` with
    ``h_0 = round(s_j r_j)``, ``h_1 = round(s_j r_j - h_0)`` in ``dtype``.

    ``scaled`` applies the per-RHS scale from ``||r_j||`` (what the solver's
    pack does with PCG state); without it ``s_j = 1``. Columns are RHS.
    """
    r = np.asarray(r, dtype=np.float64)
    r2 = r.reshape(r.shape[0], -1)
    out = np.zeros_like(r2)
    for j in range(r2.shape[1]):
        s = rhs_scale(float(np.linalg.norm(r2[:, j])), dtype) if scaled else 1.0
        v = r2[:, j] * s
        acc = np.zeros_like(v)
        for _ in range(terms):
            h = round_to(v - acc, dtype)
            acc = acc + h
        out[:, j] = acc / s
    return out.reshape(r.shape)


# Exponent of the largest scaled magnitude: |Q| <= 2**TARGET_EXP.
TARGET_EXP = {"f64": None, "f32": 0, "bf16": 0, "f16": 14}


def block_scale(amax: float, dtype: str) -> float:
    """Per-block power-of-two scale ``s`` with ``max|B/s| <= 2**TARGET_EXP``."""
    t = TARGET_EXP[dtype]
    if t is None or amax == 0.0:
        return 1.0
    e = int(np.ceil(np.log2(amax)))
    if 2.0 ** (e - 1) >= amax:  # guard log2 rounding
        e -= 1
    return float(2.0 ** (e - t))


def quantize(B: np.ndarray, dtype: str) -> tuple[float, np.ndarray]:
    """Returns ``(s, Q)`` with ``Q = round(B / s)`` in ``dtype`` (as FP64 values).
    FP64 blocks are returned as they are (scale 1, no copy)."""
    if dtype == "f64":
        return 1.0, np.asarray(B, dtype=np.float64)
    s = block_scale(float(np.max(np.abs(B))) if B.size else 0.0, dtype)
    return s, round_to(B / s, dtype)


# ---------------------------------------------------------------------------
# Schwarz preconditioners
# ---------------------------------------------------------------------------

def local_block(A: sps.csr_matrix, idx: np.ndarray) -> np.ndarray:
    return A[idx][:, idx].toarray()


def coarse_matrix(A: sps.csr_matrix, R0: sps.csr_matrix) -> np.ndarray:
    return (R0 @ A @ R0.T).toarray()


class HostCSR:
    """A SciPy CSR matrix applied through torch's CPU sparse product (threaded),
    the way the reference runs its ``CG`` on CPU tensors (``self.matrix @ p``,
    ``solvers.py:264``). ``A @ v`` for NumPy vectors / (n, R) blocks."""

    def __init__(self, A):
        import torch

        A = sps.csr_matrix(A)
        self.shape = A.shape
        self.sp = A
        with warnings.catch_warnings():  # torch flags CSR tensors as beta
            warnings.simplefilter("ignore")
            self.t = torch.sparse_csr_tensor(torch.as_tensor(A.indptr.astype(np.int64)),
                                             torch.as_tensor(A.indices.astype(np.int64)),
                                             torch.as_tensor(A.data.astype(np.float64)), A.shape)

    def __matmul__(self, v):
        import torch

        v = np.asarray(v, dtype=np.float64)
        vt = torch.from_numpy(np.ascontiguousarray(v))
        out = self.t @ (vt if vt.dim() == 2 else vt[:, None])
        return out.numpy()[:, 0] if v.ndim == 1 else out.numpy()


class Schwarz:
    """Two-level Schwarz with explicit local inverses (reference ``Inv``).

    ``batched=True`` runs the local solves the way the reference does on CPU
    tensors: the blocks of equal size stacked and applied by one batched matrix
    product (``torch.bmm``, as ``gemv_strided_batched``'s CPU counterpart) per
    size, and the sparse products through torch (``HostCSR``). Same values; the
    sums run in another order."""

    def __init__(self, A, sub_ptr, sub_idx, R0=None, block_dtype="f64", vec_dtype="f64",
                 inverse_blocks=None, batched=False):
        self.A = sps.csr_matrix(A)
        self.sub_ptr = np.asarray(sub_ptr, dtype=np.int64)
        self.sub_idx = np.asarray(sub_idx, dtype=np.int64)
        self.N = len(self.sub_ptr) - 1
        self.block_dtype = block_dtype
        self.vec_dtype = vec_dtype
        self.scales = np.ones(self.N)
        self.blocks = []
        for i in range(self.N):
            idx = self.sub_idx[self.sub_ptr[i]:self.sub_ptr[i + 1]]
            if inverse_blocks is not None:
                Binv = inverse_blocks[i]
            else:
                Ai = local_block(self.A, idx)
                Binv = np.linalg.inv(Ai) if len(idx) else np.zeros((0, 0))
            s, Q = quantize(Binv, block_dtype)
            self.scales[i] = s
            self.blocks.append(Q)
        self.R0 = None if R0 is None else sps.csr_matrix(R0)
        if self.R0 is not None:
            self.Ac = coarse_matrix(self.A, self.R0)
            self.Ac_cho = sla.cho_factor(self.Ac)
            self.AR = (self.R0 @ self.A).tocsr()
        self.groups = None
        if batched:
            self._stack()

    def _stack(self):
        """Blocks grouped by size: (sizes, stacked blocks (G, k, k), their index
        sets (G, k), scales (G)) as torch tensors; the per-block list is dropped."""
        import torch

        ks = np.diff(self.sub_ptr)
        self.groups = []
        for k in np.unique(ks):
            if k == 0:
                continue
            sel = np.nonzero(ks == k)[0]
            B = torch.from_numpy(np.stack([self.blocks[i] for i in sel]))
            idx = torch.from_numpy(np.stack([self.sub_idx[self.sub_ptr[i]:self.sub_ptr[i + 1]] for i in sel]))
            self.groups.append((B, idx, torch.from_numpy(self.scales[sel])))
            for i in sel:
                self.blocks[i] = None
        if self.R0 is not None:
            self.AR = HostCSR(self.AR)

    def _vec(self, r):
        return round_to(r, self.vec_dtype)

    def local(self, r: np.ndarray) -> np.ndarray:
        """``sum_i R_i^T (s_i Q_i) R_i r`` (columns of r are independent RHS)."""
        r = self._vec(r)
        if self.groups is not None:
            import torch

            rt = torch.from_numpy(np.ascontiguousarray(r))
            vec = rt.dim() == 1
            rt2 = rt[:, None] if vec else rt
            y = torch.zeros_like(rt2)
            for B, idx, sc in self.groups:
                Y = torch.bmm(B, rt2[idx]) * sc[:, None, None]   # (G, k, R)
                y.index_add_(0, idx.reshape(-1), Y.reshape(-1, Y.shape[-1]))
            return (y[:, 0] if vec else y).numpy()
        y = np.zeros_like(r, dtype=np.float64)
        for i in range(self.N):
            idx = self.sub_idx[self.sub_ptr[i]:self.sub_ptr[i + 1]]
            if len(idx) == 0:
                continue
            y[idx] += self.scales[i] * (self.blocks[i] @ r[idx])
        return y

    def coarse_solve(self, w):
        return sla.cho_solve(self.Ac_cho, w)

    def additive(self, r: np.ndarray) -> np.ndarray:
        y = self.local(r)
        if self.R0 is not None:
            rr = self._vec(r)
            y = y + self.R0.T @ self.coarse_solve(self.R0 @ rr)
        return self._vec(y)

    def hybrid(self, r: np.ndarray) -> np.ndarray:
        y = self.local(r)
        if self.R0 is not None:
            y = y - self.R0.T @ self.coarse_solve(self.AR @ y)
        return self._vec(y)

    def T0(self, b: np.ndarray) -> np.ndarray:
        return self.R0.T @ self.coarse_solve(self.R0 @ self._vec(b))


# ---------------------------------------------------------------------------
# PCG
# ---------------------------------------------------------------------------

def pcg(A, b, M=None, rtol=1e-7, atol=0.0, maxiter=1000, x0=None, T0=None,
        flexible=False, record_iterates=False, raise_on_fail=True):
    """Single-RHS PCG with the reference's control flow (``solvers.py:228-297``).
    ``A`` is a SciPy matrix or a ``HostCSR``."""
    A = A if isinstance(A, HostCSR) else sps.csr_matrix(A)
    b = np.asarray(b, dtype=np.float64)
    atol = max(atol, rtol * float(np.linalg.norm(b)))
    n = len(b)
    maxiter = maxiter or n * 10
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    if T0 is not None:
        x = x + T0(b)
    r = b - A @ x
    norms = []
    alphas, betas = [], []
    iterates = []
    rho_prev = None
    p = q = None
    alpha = 0.0
    i = 0
    for i in range(maxiter):
        rn = float(np.linalg.norm(r))
        norms.append(rn)
        if rn < atol:
            break
        z = M(r) if M is not None else r.copy()
        rho = float(r @ z)
        if i > 0:
            if flexible:
                beta = -alpha * float(z @ q) / rho_prev
            else:
                beta = rho / rho_prev
            p = beta * p + z
            betas.append(beta)
        else:
            p = z.copy()
        q = A @ p
        alpha = rho / float(p @ q)
        alphas.append(alpha)
        x = x + alpha * p
        r = r - alpha * q
        rho_prev = rho
        if record_iterates:
            iterates.append(x.copy())
    meta = {"iterations": len(norms) - 1, "residual norms": norms,
            "alphas": alphas, "betas": betas}
    if record_iterates:
        meta["iterates"] = iterates
    if i + 1 == maxiter and raise_on_fail:
        raise ConvergenceNotAchieved(meta)
    return x, meta


def pcg_multi(A, B, M=None, T0=None, **kw):
    """Column-by-column PCG for an ``(n, R)`` block of right-hand sides."""
    B = np.asarray(B, dtype=np.float64)
    X = np.zeros_like(B)
    its = []
    norms = []
    for j in range(B.shape[1]):
        Mj = None if M is None else (lambda r, M=M: M(r[:, None])[:, 0])
        Tj = None if T0 is None else (lambda b, T0=T0: T0(b[:, None])[:, 0])
        x, meta = pcg(A, B[:, j], Mj, T0=Tj, **kw)
        X[:, j] = x
        its.append(meta["iterations"])
        norms.append(meta["residual norms"])
    return X, {"iterations": its, "residual norms": norms}


def lanczos_condition(alphas, betas) -> float:
    """Condition-number estimate from the CG coefficients (``solvers.py:281-292``)."""
    k = len(alphas)
    L = np.zeros((k, k))
    for i in range(k):
        L[i, i] = 1.0 / alphas[i]
        if i > 0:
            L[i, i] += betas[i - 1] / alphas[i - 1]
            L[i - 1, i] = L[i, i - 1] = np.sqrt(betas[i - 1]) / alphas[i - 1]
    return float(np.linalg.cond(L, 2))


class ContiguousSchwarz:
    """Additive/hybrid Schwarz on the reference's contiguous layout.

    ``AdditiveSchwarz.solve`` (``solvers.py:811-826``): ``y = sum_i R_i^T A_i^{-1}
    R_i r + R0^T A_C^{-1} R0 r``; ``HybridSchwarz.solve`` (874-888): ``y - R0^T
    A_C^{-1} (R0 A) y``; ``HybridSchwarz.T0`` (861-872). ``R0`` sums the DOFs
    of each coarse aggregate. FP64 throughout (the plain path).
    """

    def __init__(self, A, dofs_per_solver: int, solvers_per_coarse):
        A = sps.csr_matrix(A)
        n = A.shape[0]
        k = int(dofs_per_solver)
        assert n % k == 0
        self.A, self.k, self.N = A, k, n // k
        coo = A.tocoo()
        same = (coo.row // k) == (coo.col // k)
        B = np.zeros((self.N, k, k))
        B[coo.row[same] // k, coo.row[same] % k, coo.col[same] % k] = coo.data[same]
        self.Binv = np.linalg.inv(B)
        spc = np.asarray(solvers_per_coarse, dtype=np.int64)
        owner = np.repeat(np.arange(len(spc)), spc * k)
        self.R0 = sps.csr_matrix((np.ones(n), (owner, np.arange(n))), shape=(len(spc), n))
        self.AR = (self.R0 @ A).tocsr()
        self.Ac = (self.AR @ self.R0.T).tocsc()
        self.lu = spla.splu(self.Ac)

    def local(self, r):
        import torch

        # one batched product over the equal blocks, as the reference's Inv.solve
        Y = torch.bmm(torch.from_numpy(self.Binv), torch.from_numpy(np.ascontiguousarray(r)).reshape(self.N, self.k, 1))
        return Y.reshape(-1).numpy()

    def coarse_solve(self, w):
        return self.lu.solve(w)

    def additive(self, r):
        return self.local(r) + self.R0.T @ self.coarse_solve(self.R0 @ r)

    def hybrid(self, r):
        y = self.local(r)
        return y - self.R0.T @ self.coarse_solve(self.AR @ y)

    def T0(self, b):
        return self.R0.T @ self.coarse_solve(self.R0 @ b)
