"""Host emulation of the sparse coarse-solve kernels, for tests only.

``emulate_solve`` re-runs the arithmetic of ``k_nd_gather`` / ``k_nd_fwd`` /
``k_nd_bwd`` (``dd_solvers_b200/csrc/nd.cu``) work item by work item in NumPy, with the same
index maps, level order and elimination-order buffers, so that the plan built
by ``dd_solvers_b200.nd`` can be checked without a GPU.
"""
import numpy as np

from dd_solvers_b200.nd import NDSymbolic


def emulate_solve(sym: NDSymbolic, G: np.ndarray, GT: np.ndarray, w: np.ndarray) -> np.ndarray:
    """x = A^-1 w through the plan, item by item as the kernels do."""
    n = sym.n
    w = np.asarray(w, dtype=np.float64).reshape(n, -1)
    R = w.shape[1]
    y = np.zeros((n, R))   # forward result, elimination order
    xe = np.zeros((n, R))  # solution, elimination order
    x = np.zeros((n, R))
    s_first = np.cumsum(sym.s) - sym.s
    fpos = sym.pos[sym.fidx]
    upd = np.zeros((max(sym.upd_total, 1), R))
    fb = np.full((len(sym.fidx), R), np.nan)  # gathered front vectors; NaN where never written

    def gather(t, p):
        io = int(sym.idx_off[t])
        acc = w[sym.fidx[io + p]].copy() if p < sym.s[t] else np.zeros(R)
        for q in range(sym.gptr[io + p], sym.gptr[io + p + 1]):
            acc = acc + upd[sym.gsrc[q]]
        return acc

    for lv in range(sym.n_levels):
        ga, gb = sym.gat_level_ptr[lv], sym.gat_level_ptr[lv + 1]
        for it in range(ga, gb):
            t, p0, npos = sym.gat_items[it]
            for p in range(p0, p0 + npos):
                fb[sym.idx_off[t] + p] = gather(t, p)
        for it in range(sym.fwd_level_ptr[lv], sym.fwd_level_ptr[lv + 1]):
            t, r0, nr = sym.fwd_items[it]
            s, u = int(sym.s[t]), int(sym.u[t])
            io, go = int(sym.idx_off[t]), int(sym.g_off[t])
            if gb > ga:
                f = fb[io:io + s + u]
            else:
                f = np.array([gather(t, p) for p in range(s + u)]).reshape(s + u, R)
            Gt = G[go:go + (s + u) * s].reshape(s + u, s)
            for p in range(r0, r0 + nr):
                out = Gt[p] @ f[:s] if s else np.zeros(R)
                if p < s:
                    y[s_first[t] + p] = out
                else:
                    upd[sym.upd_off[t] + p - s] = f[p] - out
    for j in range(sym.n_levels):
        for it in range(sym.bwd_level_ptr[j], sym.bwd_level_ptr[j + 1]):
            t, c0, nc = sym.bwd_items[it]
            s, u = int(sym.s[t]), int(sym.u[t])
            io, go = int(sym.idx_off[t]), int(sym.g_off[t])
            v = np.concatenate([y[s_first[t]:s_first[t] + s], -xe[fpos[io + s:io + s + u]]])
            GTt = GT[go:go + s * (s + u)].reshape(s, s + u)
            for c in range(c0, c0 + nc):
                xe[s_first[t] + c] = GTt[c] @ v
                x[sym.fidx[io + c]] = xe[s_first[t] + c]
    return x
