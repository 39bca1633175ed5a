"""ctypes binding of ``libddx.so`` (the sm_100a kernels behind ``include/ddx.h``).

The library is built in-tree by ``dd_solvers_b200/build.py`` (``__graft_entry__.build()``).
There is no fallback: if the library is missing or cannot be loaded, every
solver entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libddx.so")

# dtype codes (enum ddx_dtype)
F64, F32, BF16, F16 = 0, 1, 2, 3
DTYPE_CODE = {torch.float64: F64, torch.float32: F32, torch.bfloat16: BF16, torch.float16: F16}

# PCG state layout (ddx.h)
(ST_RHO, ST_RHO_PREV, ST_ZQ, ST_PQ, ST_ALPHA, ST_BETA, ST_RR, ST_ATOL, ST_BB, ST_T0, ST_T1, ST_ALPHA_X,
 ST_RR_PACK, ST_COUNT) = range(14)
IST_ACTIVE, IST_ITERS, IST_COUNT = range(3)
G_NACTIVE, G_MAXITER, G_FLEXIBLE, G_BREAKDOWN, G_DEFER, G_COUNT = range(6)
FIN_RZ, FIN_PQ, FIN_RR, FIN_INIT, FIN_REPLACE = range(5)
TICKETS = 16
SPMV_PLAIN, SPMV_PQ, SPMV_RES_INIT, SPMV_RES_REPLACE = range(4)

_P = C.c_void_p
_I64 = C.c_int64
_I = C.c_int
_D = C.c_double

_SIGS = {
    "ddx_last_error": (C.c_char_p, []),
    "ddx_version": (_I, []),
    "ddx_partials_len": (C.c_size_t, [_I]),
    "ddx_device_error": (_I, [C.POINTER(_I)]),
    "ddx_pcg_reset": (_I, [_I, _P, _P, _I, _I, _D, _D, _P]),
    "ddx_pcg_update_p": (_I, [_I64, _I, _P, _P, _P, _P, _P]),
    "ddx_pcg_update_px": (_I, [_I64, _I, _P, _P, _P, _P, _P, _P]),
    "ddx_pcg_flush_x": (_I, [_I64, _I, _P, _P, _P, _P, _P]),
    "ddx_pcg_update_xr": (_I, [_I64, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "ddx_pcg_finalize": (_I, [_I, _I, _P, _P, _P, _P]),
    "ddx_pcg_update_xr_pack16": (_I, [_I64, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "ddx_pcg_update_xr_pack16_ex": (_I, [_I64, _I, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P, _P]),
    "ddx_pcg_dots_rz": (_I, [_I64, _I, _P, _P, _P, _P, _P, _P, _P, _P]),
    "ddx_spmv_sell_f64": (_I, [_I64, _I64, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P, _P]),
    "ddx_spmv_csr_f64": (_I, [_I64, _I, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P, _P]),
    "ddx_spmv_csr_ordered_f64": (_I, [_I64, _I, _P, _P, _P, _P, _I, _P, _P, _P, _I, _P, _P, _P, _P, _P, _P]),
    "ddx_row_clusters": (_I, [_I64, _P, _P, _I, _P]),
    "ddx_spmv_csr_rowblock_mapped": (_I, [_I64, _I, _P, _P, _P, _P, _P, _P, _I, _P, _P]),
    "ddx_spmv_csr_rowblock_f64": (_I, [_I64, _I, _P, _P, _P, _P, _P, _P]),
    "ddx_spmv_bsr": (_I, [_I64, _I, _P, _P, _P, _P, _P, _I, _P]),
    "ddx_spmv_epilogue_f64": (_I, [_I64, _P, _P, _P, _I, _P, _P, _P, _P, _P, _P]),
    "ddx_gemv_strided_batched": (_I, [_I64, _I, _P, _I, _P, _P, _I, _P]),
    "ddx_schwarz_local_apply": (_I, [_I, _I, _P, _P, _P, _P, _P, _I, _P, _I, _P, _P, _I, _P, _P]),
    "ddx_schwarz_local_apply_ex": (_I, [_I, _I, _P, _P, _P, _P, _P, _I, _P, _I, _P, _P, _I, _P, _I, _I, _P]),
    "ddx_schwarz_local_apply_sym": (_I, [_I, _I, _P, _P, _P, _P, _P, _I, _P, _I, _P, _P, _I, _P, _I, _I, _I, _P]),
    "ddx_schwarz_local_apply_tc_sym": (_I, [_I, _I, _P, _P, _P, _P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _P]),
    "ddx_schwarz_local_apply_tc": (_I, [_I, _I, _P, _P, _P, _P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _P]),
    "ddx_schwarz_local_apply_tc_sym_ex": (_I, [_I, _I, _P, _P, _P, _P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _I, _P]),
    "ddx_dot_noalloc": (_I, [_I64, _I, _P, _P, _P, _P]),
    "ddx_pack_panels16": (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _I, _I, _P]),
    "ddx_schwarz_combine": (_I, [_I64, _I, _P, _P, _P, _I, _P, _P, _P, _P, _P, _D, _P, _I, _P, _P, _P, _P,
                                 _P, _P, _P]),
    "ddx_coarse_gemv_f64": (_I, [_I, _I, _P, _P, _P, _P, _P]),
    "ddx_coarse_gemm_f64": (_I, [_I, _I, _P, _P, _P, _P, _I64, _P, _P]),
    "ddx_schwarz_combine_update": (_I, [_I64, _I, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P, _D, _P, _P, _P, _P,
                                        _P]),
    "ddx_schwarz_combine_ex": (_I, [_I64, _I, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P, _D, _P, _I, _P, _P, _P, _P,
                                    _P, _P, _P]),
    "ddx_schwarz_restrict_sub": (_I, [_I, _I64, _I64, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I64, _P,
                                      _P, _P, _P, _P, _P]),
    "ddx_nd_order": (_I, [_I64, _P, _P, _I, _P, _P, _P, _P]),
    "ddx_spmv_csr_lanes_f64": (_I, [_I64, _I, _P, _P, _P, _P, _P, _P]),
    "ddx_spmv_csr_lanes": (_I, [_I64, _I, _P, _P, _P, _P, _I, _P, _P]),
    "ddx_schwarz_local_apply_small": (_I, [_I, _I, _P, _P, _P, _P, _I, _P, _I, _I, _I64, _P, _P, _I, _P, _P]),
    "ddx_coarse_solve_nd": (_I, [_P, _I, _P, _P, _P, _P, _P, _P, _P, _P]),
    "ddx_nd_update_sets": (_I, [_I64, _I64, _P, _P, _P, _P, _P, _P, _P, _I64, _P]),
    "ddx_elem_grad_q1": (_I, [_I, _I, _P, _P, _P, _P, _P]),
}

_lib = None


class DDXError(RuntimeError):
    pass


def lib() -> C.CDLL:
    """Loads the library once; raises if it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise DDXError(
                f"CUDA library {LIB_PATH} is missing: run dd_solvers_b200.build.build() "
                "(or __graft_entry__.build()) first")
        torch.cuda.init() if torch.cuda.is_available() else None
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


# Number of library calls issued (each launches one kernel; the local apply
# launches one per right-hand side). CUDA-graph replays add their captured count.
CALLS = [0]


def call(name: str, *args) -> None:
    CALLS[0] += 1
    status = getattr(lib(), name)(*args)
    if status != 0:
        msg = lib().ddx_last_error().decode()
        raise DDXError(f"{name} failed (status {status}): {msg}")


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    return t.data_ptr()


def stream_ptr() -> int:
    return torch.cuda.current_stream().cuda_stream


def device_error() -> int:
    code = C.c_int(0)
    call("ddx_device_error", C.byref(code))
    return code.value


def require_cuda(t: torch.Tensor, what: str) -> None:
    if not t.is_cuda:
        raise DDXError(f"{what} must be a CUDA tensor (this package has no CPU path)")
