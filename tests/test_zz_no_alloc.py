"""ddx_dot_noalloc: the dot-product entry point that needs no caller scratch.

It exists for callers that cannot allocate device memory when they need a dot
product (behind a plain C FFI without a device allocator, or in loops that must
not allocate after start-up). This test
calls it through the C ABI twice in a row and checks each result against the
existing entry point, ddx_pcg_dots_rz (which takes caller-allocated scratch),
on the same inputs. It is collected last so a failure here cannot hide
failures elsewhere, and it passes both alone and after the other tests.
"""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu


def _noalloc():
    from dd_solvers_b200 import _lib

    f = _lib.lib().ddx_dot_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return f


def _reference_dots(x, y, n, R):
    """rho_j = x_j . y_j through ddx_pcg_dots_rz with freshly allocated scratch."""
    from dd_solvers_b200 import _lib as L

    dev = x.device
    st = torch.zeros(L.ST_COUNT * R, dtype=torch.float64, device=dev)
    ist = torch.zeros(L.IST_COUNT * R + L.G_COUNT, dtype=torch.int32, device=dev)
    partials = torch.zeros(int(L.lib().ddx_partials_len(R)), dtype=torch.float64, device=dev)
    tickets = torch.zeros(L.TICKETS, dtype=torch.int32, device=dev)
    L.call("ddx_pcg_reset", R, L.ptr(st), L.ptr(ist), 10, 0, 1e-8, 0.0, L.stream_ptr())
    L.call("ddx_pcg_dots_rz", n, R, L.ptr(x), L.ptr(y), None, L.ptr(st), L.ptr(ist), L.ptr(partials),
           L.ptr(tickets), L.stream_ptr())
    return st.view(L.ST_COUNT, R)[L.ST_RHO].clone()


@pytest.mark.parametrize("n,R", [(1, 1), (300_001, 1), (100_000, 8), (50_003, 64)])
def test_dot_noalloc_matches_scratch_entry_point_twice(cuda, n, R):
    from dd_solvers_b200 import _lib as L

    f = _noalloc()
    gen = torch.Generator(device=cuda).manual_seed(n + R)
    for call in range(2):  # the shared array keeps the previous call's contents
        x = torch.randn(n * R, dtype=torch.float64, device=cuda, generator=gen)
        y = torch.randn(n * R, dtype=torch.float64, device=cuda, generator=gen)
        out = torch.full((R,), float("nan"), dtype=torch.float64, device=cuda)
        status = f(n, R, x.data_ptr(), y.data_ptr(), out.data_ptr(), L.stream_ptr())
        assert status == 0, L.lib().ddx_last_error()
        ref = _reference_dots(x, y, n, R)
        torch.cuda.synchronize()
        assert torch.allclose(out, ref, rtol=1e-12, atol=1e-12 * float(ref.abs().max())), (call, out, ref)


def test_dot_noalloc_rejects_too_many_rhs(cuda):
    from dd_solvers_b200 import _lib as L

    f = _noalloc()
    x = torch.zeros(128, dtype=torch.float64, device=cuda)
    out = torch.zeros(128, dtype=torch.float64, device=cuda)
    assert f(1, 128, x.data_ptr(), x.data_ptr(), out.data_ptr(), L.stream_ptr()) == 1
    assert b"R=128" in L.lib().ddx_last_error()


def test_dot_noalloc_rejects_bad_arguments_and_allocates_nothing(cuda):
    """A null pointer or n < 0 is refused with status 1; after a first call on
    the device, further calls leave torch's allocator and the device's free
    memory unchanged."""
    from dd_solvers_b200 import _lib as L

    f = _noalloc()
    x = torch.ones(1000, dtype=torch.float64, device=cuda)
    out = torch.zeros(1, dtype=torch.float64, device=cuda)
    assert f(1000, 1, None, x.data_ptr(), out.data_ptr(), L.stream_ptr()) == 1
    assert f(-1, 1, x.data_ptr(), x.data_ptr(), out.data_ptr(), L.stream_ptr()) == 1
    assert f(1000, 1, x.data_ptr(), x.data_ptr(), out.data_ptr(), L.stream_ptr()) == 0
    torch.cuda.synchronize()
    alloc, reserved = torch.cuda.memory_allocated(cuda), torch.cuda.memory_reserved(cuda)
    free0 = torch.cuda.mem_get_info(cuda)[0]
    for _ in range(3):
        assert f(1000, 1, x.data_ptr(), x.data_ptr(), out.data_ptr(), L.stream_ptr()) == 0
    torch.cuda.synchronize()
    assert float(out[0]) == 1000.0
    assert torch.cuda.memory_allocated(cuda) == alloc and torch.cuda.memory_reserved(cuda) == reserved
    assert abs(torch.cuda.mem_get_info(cuda)[0] - free0) <= 1 << 20
