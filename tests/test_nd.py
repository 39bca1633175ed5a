"""Nested-dissection multifrontal coarse solver: ordering, symbolic analysis
and numeric factorisation on the host, and the solve kernels' arithmetic
emulated item by item (``tests/nd_emulation.py``) against SciPy's sparse LU."""
import os
import sys

import numpy as np
import pytest
import scipy.sparse as sps
import scipy.sparse.linalg as spla

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from dd_solvers_b200 import dg, nd  # noqa: E402
from nd_emulation import emulate_solve  # noqa: E402


def lap2d(k, shift=0.01):
    T = sps.diags([-1, 2, -1], [-1, 0, 1], shape=(k, k))
    return (sps.kron(sps.eye(k), T) + sps.kron(T, sps.eye(k)) + shift * sps.eye(k * k)).tocsr()


def random_spd(n, density, seed):
    B = sps.random(n, n, density=density, random_state=seed)
    return (B + B.T + 10 * sps.eye(n)).tocsr()


def dg_p0_coarse(m, solver_level):
    s = dg.sipg_p1(dg.uniform_mesh_2d(m))
    A = sps.csr_matrix((s.matrix.values().numpy(), s.matrix.col_indices().numpy(),
                        s.matrix.crow_indices().numpy()), shape=tuple(s.matrix.shape))
    n = A.shape[0]
    k = 3 * 4 ** (m - solver_level)
    R0 = sps.csr_matrix((np.ones(n), (np.arange(n) // k, np.arange(n))), shape=(n // k, n))
    return (R0 @ A @ R0.T).tocsr()


CASES = {
    "grid20": lambda: lap2d(20),
    "grid45": lambda: lap2d(45),
    "random_disconnected": lambda: random_spd(300, 0.01, 1),
    "dg_p0_S7_on_S4": lambda: dg_p0_coarse(7, 4),
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("leaf,top_merge,small_items", [(8, None, False), (64, None, False), (16, 0, True)])
def test_emulated_solve_matches_sparse_lu(case, leaf, top_merge, small_items):
    """The last variant keeps the whole separator tree and cuts 8-row items,
    so the upper levels run the gather launch."""
    A = CASES[case]()
    A.sort_indices()
    sym = nd.NDSymbolic(A.indptr, A.indices, A.shape[0], leaf, top_merge)
    if small_items:
        sym.build_items(512, 8)
    G, GT = (t.numpy() for t in nd.factorize(sym, A.indptr, A.indices, A.data, "cpu"))
    w = np.random.default_rng(0).standard_normal((A.shape[0], 3))
    x = emulate_solve(sym, G, GT, w)
    ref = spla.splu(A.tocsc()).solve(w)
    assert np.abs(x - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("case", sorted(CASES))
def test_ordering_is_a_postorder_separator_tree(case):
    A = CASES[case]()
    n = A.shape[0]
    S, parent = nd.nested_dissection(A.indptr, A.indices, n, 16)
    perm = np.concatenate(S)
    assert np.array_equal(np.sort(perm), np.arange(n))
    nf = len(S)
    assert all(parent[t] == -1 or parent[t] > t for t in range(nf))  # children first
    # no edge joins two different subtrees without passing an ancestor: an
    # edge (i, j) is allowed only if one endpoint's node is an ancestor of
    # (or equal to) the other's
    node_of = np.empty(n, dtype=np.int64)
    for t, s in enumerate(S):
        node_of[s] = t

    def ancestors(t):
        out = set()
        while t >= 0:
            out.add(t)
            t = parent[t]
        return out

    anc = [ancestors(t) for t in range(nf)]
    coo = A.tocoo()
    for i, j in zip(coo.row, coo.col):
        a, b = node_of[i], node_of[j]
        assert a in anc[b] or b in anc[a]


def test_symbolic_front_sets():
    A = lap2d(30)
    sym = nd.NDSymbolic(A.indptr, A.indices, A.shape[0], 32)
    for t in range(sym.nf):
        assert len(sym.S[t]) >= 1
        # the update set follows the separator in elimination order
        if len(sym.U[t]):
            assert sym.pos[sym.U[t]].min() > sym.pos[sym.S[t]].max()
        if sym.parent[t] < 0:
            assert len(sym.U[t]) == 0
    # the forward items cover each front's rows, the backward items its columns, once
    for items, total in ((sym.fwd_items, sym.s + sym.u), (sym.bwd_items, sym.s)):
        rows = {}
        for t, r0, nr in items:
            rows.setdefault(int(t), []).append((int(r0), int(nr)))
        for t in range(sym.nf):
            cover = sorted(rows[t])
            ends = [r0 + nr for r0, nr in cover]
            assert cover[0][0] == 0 and ends[-1] == total[t]
            assert all(cover[i + 1][0] == ends[i] for i in range(len(cover) - 1))


@pytest.mark.parametrize("case", ["grid45", "dg_p0_S7_on_S4"])
def test_gather_items_cover_their_levels(case):
    """Where a level has gather items, they cover every position of every
    front of that level exactly once; levels whose fronts are cut into many
    forward items get them."""
    A = CASES[case]()
    sym = nd.NDSymbolic(A.indptr, A.indices, A.shape[0], 16, top_merge=0)
    sym.build_items(512, 8)
    m = sym.s + sym.u
    gathered = 0
    for lv in range(sym.n_levels):
        ga, gb = sym.gat_level_ptr[lv], sym.gat_level_ptr[lv + 1]
        a, b = sym.fwd_level_ptr[lv], sym.fwd_level_ptr[lv + 1]
        repeated = int(sym.s[sym.fwd_items[a:b, 0]].sum())
        once = int(m[sym.by_level[lv]].sum())
        assert (gb > ga) == (lv >= nd.GATHER_MIN_LEVEL and repeated >= nd.GATHER_MIN_RATIO * once)
        if gb == ga:
            continue
        gathered += 1
        cover = {}
        for t, p0, npos in sym.gat_items[ga:gb]:
            assert 0 < npos <= nd.GATHER_POSITIONS
            cover.setdefault(int(t), []).append((int(p0), int(npos)))
        assert sorted(cover) == sorted(int(t) for t in sym.by_level[lv])
        for t, parts in cover.items():
            parts.sort()
            assert parts[0][0] == 0 and parts[-1][0] + parts[-1][1] == m[t]
            assert all(parts[i][0] + parts[i][1] == parts[i + 1][0] for i in range(len(parts) - 1))
    assert gathered >= 1


def test_plan_binding_matches_the_c_struct(tmp_path):
    """``nd._Plan`` (ctypes) has the layout of ``ddx_nd_plan`` in
    ``include/ddx.h``: every field at the same offset, the same size."""
    import ctypes
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    names = [f[0] for f in nd._Plan._fields_]
    src = tmp_path / "plan_layout.c"
    body = "".join(f'  printf("{n} %zu\\n", offsetof(ddx_nd_plan, {n}));\n' for n in names)
    src.write_text("#include <stddef.h>\n#include <stdio.h>\n#include \"ddx.h\"\nint main(void) {\n"
                   + body + '  printf("sizeof %zu\\n", sizeof(ddx_nd_plan));\n  return 0;\n}\n')
    exe = tmp_path / "plan_layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                       text=True).stdout.splitlines())
    for n in names:
        assert int(out[n]) == getattr(nd._Plan, n).offset, n
    assert int(out["sizeof"]) == ctypes.sizeof(nd._Plan)


def test_solver_size_switches(monkeypatch):
    """The size rules of ``nd.NDSolver`` (built on the host here, no solve):
    up to ``OVERLAP_MAX_N`` rows the sweeps stage their operator rows, gather
    per front and release the next level early; above ``FAT_ITEMS_MIN_N``
    the items are re-cut to 64 KB."""
    import torch

    A = lap2d(45)
    A.sort_indices()
    At = torch.sparse_csr_tensor(torch.as_tensor(A.indptr), torch.as_tensor(A.indices), torch.as_tensor(A.data),
                                 A.shape)
    s = nd.NDSolver(At, leaf=16, top_merge=0)
    assert s.gather and s.plan.release_early == 1
    assert np.array_equal(s.fwd_level_gmax, s.sym.fwd_level_gmax)
    small = s.sym.fwd_items.shape[0]
    monkeypatch.setattr(nd, "OVERLAP_MAX_N", 100)
    monkeypatch.setattr(nd, "FAT_ITEMS_MIN_N", 100)
    s = nd.NDSolver(At, leaf=16, top_merge=0)
    assert not s.gather and s.plan.release_early == 0
    assert (s.fwd_level_gmax < 0).all() and (s.bwd_level_gmax < 0).all()
    assert s.sym.fwd_items.shape[0] <= small
    assert int(s.sym.fwd_items[:, 2].max()) <= 128


def test_threaded_ordering_matches_single_threaded(monkeypatch):
    """The ordering runs the halves below large separators on separate
    threads; the separator tree and permutation are the same for any thread
    count (40,000 vertices: halves above the threading threshold)."""
    A = lap2d(200)
    A.sort_indices()
    out = []
    for threads in ("1", "2", "8"):
        monkeypatch.setenv("DDX_ND_THREADS", threads)
        S, parent = nd.nested_dissection(A.indptr, A.indices, A.shape[0], 64)
        out.append((np.concatenate(S), np.array([len(x) for x in S]), parent))
    for perm, sizes, parent in out[1:]:
        assert np.array_equal(perm, out[0][0])
        assert np.array_equal(sizes, out[0][1])
        assert np.array_equal(parent, out[0][2])


def test_update_sets_native_contract():
    """``ddx_nd_update_sets`` on a two-front tree (a 2 x 2 full matrix, one
    vertex per front): U_0 = {1}, U_1 = {}; a capacity below the total is
    refused with the total reported, then the call succeeds."""
    from dd_solvers_b200 import _lib as L

    i64 = lambda *v: np.array(v, dtype=np.int64)  # noqa: E731
    s_first, s_size, p_ptr, p_pos, parent = i64(0, 1), i64(1, 1), i64(0, 2, 4), i64(0, 1, 0, 1), i64(1, -1)
    u_ptr = np.zeros(3, dtype=np.int64)
    u_pos = np.zeros(1, dtype=np.int64)
    total = np.zeros(1, dtype=np.int64)
    args = [x.ctypes.data for x in (s_first, s_size, p_ptr, p_pos, parent, u_ptr, u_pos)]
    with pytest.raises(L.DDXError):
        L.call("ddx_nd_update_sets", 2, 2, *args, 0, total.ctypes.data)
    assert total[0] == 1
    L.call("ddx_nd_update_sets", 2, 2, *args, 1, total.ctypes.data)
    assert list(u_ptr) == [0, 1, 1] and list(u_pos) == [1]


def _update_sets_numpy(s_first, s_size, p_ptr, p_pos, parent):
    """The update-set rule restated with numpy, front by front: the positions
    after the front's separator reached by its rows or by its children's update
    sets, sorted and distinct (np.unique)."""
    nf = len(s_size)
    sets = []
    children = [[] for _ in range(nf)]
    for t in range(nf):
        if parent[t] >= 0:
            children[parent[t]].append(t)
    for t in range(nf):
        last = s_first[t] + s_size[t] - 1
        parts = [p_pos[p_ptr[s_first[t]]:p_ptr[s_first[t] + s_size[t]]]] + [sets[c] for c in children[t]]
        u = np.unique(np.concatenate(parts)) if parts else np.zeros(0, dtype=np.int64)
        sets.append(u[u > last])
    u_ptr = np.concatenate([[0], np.cumsum([len(x) for x in sets])]).astype(np.int64)
    u_pos = np.concatenate(sets) if sets else np.zeros(0, dtype=np.int64)
    return u_ptr, u_pos


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("top_merge", [0, 64])
def test_update_sets_native_equal_numpy(name, top_merge):
    """``ddx_nd_update_sets`` returns exactly the numpy restatement's sets
    (same pointers, same sorted positions) on every ordering case, with and
    without the merged top front."""
    A = CASES[name]()
    A = sps.csr_matrix(A)
    A.sort_indices()
    n = A.shape[0]
    S, parent = nd.nested_dissection(A.indptr, A.indices, n, 16)
    S, parent = nd._merge_top(S, parent, top_merge)
    perm = np.concatenate(S)
    pos = np.empty(n, dtype=np.int64)
    pos[perm] = np.arange(n)
    s_size = np.array([len(x) for x in S], dtype=np.int64)
    s_first = np.concatenate([[0], np.cumsum(s_size)[:-1]]).astype(np.int64)
    indptr = A.indptr.astype(np.int64)
    deg = np.diff(indptr)[perm]
    p_ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(deg, out=p_ptr[1:])
    p_idx = A.indices.astype(np.int64)[np.repeat(indptr[perm] - p_ptr[:-1], deg) + np.arange(int(p_ptr[-1]))]
    p_pos = pos[p_idx]
    u_ptr, u_pos = nd._update_sets(n, s_first, s_size, p_ptr, p_pos, parent)
    r_ptr, r_pos = _update_sets_numpy(s_first, s_size, p_ptr, p_pos, parent)
    assert np.array_equal(u_ptr, r_ptr)
    assert np.array_equal(u_pos, r_pos)


def test_update_sets_rejects_bad_fronts():
    """A front table whose separator range leaves [0, n), or a decreasing
    p_ptr, is refused with a status (no out-of-range host reads)."""
    from dd_solvers_b200 import _lib as L

    i64 = lambda *v: np.array(v, dtype=np.int64)  # noqa: E731
    p_ptr, p_pos, parent = i64(0, 2, 4), i64(0, 1, 0, 1), i64(1, -1)
    u_ptr = np.zeros(3, dtype=np.int64)
    u_pos = np.zeros(4, dtype=np.int64)
    total = np.zeros(1, dtype=np.int64)
    for s_first, s_size, pp in ((i64(0, 1), i64(1, 2), p_ptr), (i64(-1, 1), i64(1, 1), p_ptr),
                                (i64(0, 1), i64(1, 1), i64(0, 3, 2))):
        args = [x.ctypes.data for x in (s_first, s_size, pp, p_pos, parent, u_ptr, u_pos)]
        with pytest.raises(L.DDXError):
            L.call("ddx_nd_update_sets", 2, 2, *args, 4, total.ctypes.data)
