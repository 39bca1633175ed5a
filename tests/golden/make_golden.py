"""Writes the golden fixtures under tests/golden/ from the reference itself.

Run with DDX_REFERENCE_ROOT set to a checkout of the reference:
    DDX_REFERENCE_ROOT=<reference checkout>  python tests/golden/make_golden.py

* fixture24.npz  - the 24-DOF DG-SIPG system of the reference's solver test
                   (src/dd_solvers/tests/test_solvers.py:25-108) and the
                   reference's own CG/AdditiveSchwarz/HybridSchwarz results on
                   it (run on CPU through oracle/ref_harness.py).
* c1r.npz        - "config 1-R": 2D Q1 Poisson on 256x256 cells (255^2 DOFs),
                   U[-1,1] load vector (seed 0), 15x15 equal subdomains of 17^2
                   DOFs, one P0 aggregate each; the reference's ASM/HSM FP64
                   iteration counts, residual histories and solutions.
* unit_cases.npz - known-answer inputs/outputs captured while running the
                   reference's own unit tests for sort_csr / gather_csr
                   (tests/test_cusparse.py), spd_factorize (tests/test_cudss.py),
                   the BSR fixture (tests/test_bsr.py:9-138) and the condition
                   number estimate (tests/test_solvers.py:179-184).
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref_harness  # noqa: E402

S = ref_harness.load()
import numpy as np  # noqa: E402
import torch  # noqa: E402

from dd_solvers_b200 import partition, problems  # noqa: E402

REF = ref_harness.REF_ROOT
TESTS = os.path.join(REF, "src", "dd_solvers", "tests")


def _exec_slice(path, start_marker, end_marker):
    src = open(path).read()
    a, b = src.index(start_marker), src.index(end_marker)
    ns = {}
    exec("import torch\n" + src[a:b], ns)
    return ns


def _csr_np(t):
    return (t.crow_indices().numpy().astype(np.int64), t.col_indices().numpy().astype(np.int64),
            t.values().numpy().astype(np.float64))


def run_cg(A, b, pc, rtol, maxiter=1000, **setup_kw):
    cg = S.CG(pc, rtol=rtol, maxiter=maxiter, bsr_matmul=False)
    cg.setup(A, **setup_kw)
    x, meta = cg.solve(b)
    return x.numpy().astype(np.float64), meta


def fixture24():
    ns = _exec_slice(os.path.join(TESTS, "test_solvers.py"), "form_matrix =", "device = torch.device")
    A = ns["form_matrix"].double()
    b = ns["load_vector"].double()
    f2s, s2c = ns["fine_to_solvers"], ns["solvers_to_coarse"]
    f2d = torch.arange(24, dtype=torch.int32).reshape(8, 3)
    n_coarse = int(s2c.max()) + 1
    spc = s2c.bincount(minlength=n_coarse)
    perm = S.asm_permutation(fine_to_solvers=f2s, solvers_to_coarse=s2c, fine_to_dofs=f2d)
    inv = S.inverse_permutation(perm)
    Ap = S.permute_csr_tensor(A, inv)
    out = {"crow": _csr_np(A)[0], "col": _csr_np(A)[1], "val": _csr_np(A)[2], "load": b.numpy(),
           "fine_to_solvers": f2s.numpy(), "solvers_to_coarse": s2c.numpy(), "perm": perm.numpy(),
           "p_crow": _csr_np(Ap)[0], "p_col": _csr_np(Ap)[1], "p_val": _csr_np(Ap)[2]}
    rng = np.random.default_rng(24)
    b2 = torch.as_tensor(rng.uniform(-1, 1, 24))
    out["rhs_u"] = b2.numpy()
    cases = {
        "asm_f64": lambda: S.AdditiveSchwarz(torch.float64, S.Inv(), S.CUDSS()),
        "hsm_f64": lambda: S.HybridSchwarz(torch.float64, S.Inv(), S.CUDSS()),
        "asm_f64_inv32": lambda: S.AdditiveSchwarz(torch.float64, S.Inv(torch.float32), S.CUDSS()),
        "hsm_f64_inv32": lambda: S.HybridSchwarz(torch.float64, S.Inv(torch.float32), S.CUDSS()),
        "none": lambda: None,
    }
    for rhs_name, rhs in (("load", b), ("rhs_u", b2)):
        for name, mk in cases.items():
            x, meta = run_cg(Ap, rhs[perm], mk(), rtol=1e-12, dofs_per_solver=6, solvers_per_coarse=spc,
                             block_size=3)
            key = f"{rhs_name}__{name}"
            out[key + "__x"] = x
            out[key + "__iters"] = np.array(meta["iterations"])
            out[key + "__norms"] = np.array(meta["residual norms"])
    np.savez_compressed(os.path.join(HERE, "fixture24.npz"), **out)
    print("fixture24:", {k: int(v) for k, v in out.items() if k.endswith("__iters")})


def c1r():
    P = problems.poisson2d(256)
    A = P.matrix
    n = A.shape[0]
    b = problems.uniform_rhs(n, seed=0)
    owner, nparts = partition.box_owner(P.interior_shape, 15)
    # 255 = 15 * 17: box_owner on 256 cells with 15 parts gives 17-node boxes
    counts = np.bincount(owner, minlength=nparts)
    assert np.all(counts == 289), counts
    perm = np.argsort(owner, kind="stable")  # new position -> old DOF
    inv = np.empty(n, dtype=np.int64)
    inv[perm] = np.arange(n)
    At = torch.sparse_csr_tensor(torch.as_tensor(A.indptr.astype(np.int64)), torch.as_tensor(A.indices.astype(np.int64)),
                                 torch.as_tensor(A.data), A.shape)
    Ap = S.permute_csr_tensor(At, torch.as_tensor(inv))
    bp = torch.as_tensor(b[perm])
    spc = torch.ones(nparts, dtype=torch.int64)
    # b and perm are regenerated from the seed in the tests; keep a fingerprint of b
    out = {"b_head": b[:16].copy(), "b_sum": np.array(b.sum()), "perm_head": perm[:64].copy()}
    for name, mk in (("asm_f64", lambda: S.AdditiveSchwarz(torch.float64, S.Inv(), S.CUDSS())),
                     ("hsm_f64", lambda: S.HybridSchwarz(torch.float64, S.Inv(), S.CUDSS()))):
        x, meta = run_cg(Ap, bp, mk(), rtol=1e-8, dofs_per_solver=289, solvers_per_coarse=spc, block_size=1)
        out[name + "__x"] = x
        out[name + "__iters"] = np.array(meta["iterations"])
        out[name + "__norms"] = np.array(meta["residual norms"])
        print("c1r", name, meta["iterations"])
    np.savez_compressed(os.path.join(HERE, "c1r.npz"), **out)


def unit_cases():
    out = {}
    # --- sort_csr / gather_csr: run the reference tests against the harness ops and record pairs
    calls = []
    cus = sys.modules["ddref.cusparse"]

    def rec(fn, tag):
        def wrapped(m, *a, **k):
            res = fn(m, *a, **k)
            calls.append((tag, m, res))
            return res
        return wrapped

    fake = types.ModuleType("dd_solvers.cusparse")
    fake.sort_csr = rec(cus.sort_csr, "sort")
    fake.gather_csr = rec(cus.gather_csr, "gather")
    sys.modules["dd_solvers"] = types.ModuleType("dd_solvers")
    sys.modules["dd_solvers.cusparse"] = fake
    spec = importlib.util.spec_from_file_location("ref_test_cusparse", os.path.join(TESTS, "test_cusparse.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.device = torch.device("cpu")
    for dt in (torch.float64,):
        mod.test_sort_csr(torch.int64, dt, 1)
    mod.test_gather_csr_simple()
    mod.test_gather_csr_empty_row()
    for i, (tag, m, res) in enumerate(calls):
        for part, (cr, co, va) in (("in", _csr_np(m)), ("out", _csr_np(res))):
            out[f"{tag}{i}_{part}_crow"], out[f"{tag}{i}_{part}_col"], out[f"{tag}{i}_{part}_val"] = cr, co, va
    out["n_cusparse_cases"] = np.array(len(calls))

    # --- spd_factorize known answers (tests/test_cudss.py:12-84)
    src_c = open(os.path.join(TESTS, "test_cudss.py")).read()
    a, b_ = src_c.index("    # 2 0 2"), src_c.index("@pytest.mark.parametrize")
    block = "\n".join(l[4:] if l.startswith("    ") else l for l in src_c[a:b_].splitlines())
    ns = {"torch": torch, "device": "cpu"}
    exec(block, ns)
    for name in ("spd_3x3", "spd_2x2"):
        t = ns[name]
        cr, co, va = _csr_np(t)
        out[name + "_crow"], out[name + "_col"], out[name + "_val"] = cr, co, va
    src = open(os.path.join(TESTS, "test_cudss.py")).read()
    # solutions / right-hand sides as written in the test
    env = {"torch": torch, "device": "cpu"}
    for line in src.splitlines():
        s = line.strip()
        if s.startswith(("x1 =", "x2 =", "b1 =", "b2 =", "x =", "b =")) and "torch.tensor" in s:
            name = s.split("=")[0].strip()
            vt = torch.float64
            env["value_type"] = vt
            val = eval(s.split("=", 1)[1], env)
            out["cudss_" + name] = val.numpy().astype(np.float64)

    # --- BSR fixture (tests/test_bsr.py:9-138)
    nsb = _exec_slice(os.path.join(TESTS, "test_bsr.py"), "matrix = torch.sparse_bsr_tensor(", "def allclose")
    mb = nsb["matrix"]
    out["bsr_crow"] = mb.crow_indices().numpy()
    out["bsr_col"] = mb.col_indices().numpy()
    out["bsr_val"] = mb.values().numpy().astype(np.float64)
    out["bsr_dense"] = mb.to_dense().numpy().astype(np.float64)

    # --- condition number estimate (tests/test_solvers.py:179-184), reference CG on CPU
    cg = S.CG(preconditioner=None, rtol=1e-9, estimate_cond=True, bsr_matmul=False)
    cg.setup(torch.diag(torch.tensor([0.5, 4, 21])).to_sparse_csr())
    _, meta = cg.solve(torch.ones(3))
    out["cond_estimate"] = np.array(meta["condition number estimate"])
    out["cond_iters"] = np.array(meta["iterations"])
    np.savez_compressed(os.path.join(HERE, "unit_cases.npz"), **out)
    print("unit cases: cusparse", len(calls), "cond", float(out["cond_estimate"]))


if __name__ == "__main__":
    fixture24()
    unit_cases()
    c1r()
