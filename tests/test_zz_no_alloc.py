"""tval3g_dense_adjoint_static: y = A^T x with no device allocation.

It serves callers that cannot allocate device memory when they call in (their
device memory is reserved up front by another allocator, or a cudaMalloc's
synchronisation is not acceptable).  Its scratch is a fixed array inside the
library, shared by all calls.  This file runs last (pytest collects files in
name order) and also passes alone in a fresh process.

Checked against the regular dense operator entry point (tval3g_op_apply,
trans = 1) within the operator tolerance of the suite (1e-5 relative), on two
calls in a row with different inputs, so stale scratch would show; the calls
run on a non-default stream (the entry point is stream-ordered), and a warm
call leaves the device's free memory unchanged.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import relerr
from tval3g import capi

pytestmark = pytest.mark.gpu


def _static_adjoint(A_dev, m, n, x_dev, y_dev, stream=None):
    L = capi.lib()
    f = L.tval3g_dense_adjoint_static
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    return f(A_dev.data_ptr(), m, n, x_dev.data_ptr(), y_dev.data_ptr(), stream)


@pytest.mark.parametrize("m,n", [(1229, 4096), (307, 1021)])
def test_static_adjoint_matches_operator(m, n, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(m + n)
    A = (rng.standard_normal((m, n)) / np.sqrt(m)).astype(np.float32)
    A_dev = torch.tensor(A, device="cuda")
    op = capi.Operator(capi.dense_problem((1, n), A))
    side = torch.cuda.Stream()
    for call in range(2):
        x = torch.tensor(rng.standard_normal(m).astype(np.float32), device="cuda")
        want = torch.empty(n, device="cuda")
        op.apply(x, want, trans=True)
        got = torch.full((n,), float("nan"), device="cuda")
        torch.cuda.synchronize()
        assert _static_adjoint(A_dev, m, n, x, got, side.cuda_stream) == capi.OK, capi.lib().tval3g_last_error()
        side.synchronize()
        e_op = relerr(got.cpu().numpy(), want.cpu().numpy())
        ref = A.astype(np.float64).T @ x.cpu().numpy().astype(np.float64)
        e_64 = relerr(got.cpu().numpy(), ref)
        print(f"m={m} n={n} call {call}: vs tval3g_op_apply {e_op:.2e}, vs FP64 {e_64:.2e}")
        assert e_op < 1e-5, call
        assert e_64 < 1e-5
    op.close()


def test_static_adjoint_allocates_nothing_when_warm(torch_cuda):
    torch = torch_cuda
    m, n = 1229, 4096
    rng = np.random.default_rng(3)
    A_dev = torch.tensor((rng.standard_normal((m, n)) / np.sqrt(m)).astype(np.float32), device="cuda")
    x = torch.tensor(rng.standard_normal(m).astype(np.float32), device="cuda")
    y = torch.empty(n, device="cuda")
    assert _static_adjoint(A_dev, m, n, x, y) == capi.OK   # the first call on the device (set-up)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert _static_adjoint(A_dev, m, n, x, y) == capi.OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_static_adjoint_rejects_oversize(torch_cuda):
    torch = torch_cuda
    n = (1 << 20) + 1
    A = torch.zeros(1, device="cuda")
    x = torch.zeros(1, device="cuda")
    y = torch.zeros(1, device="cuda")
    rc = _static_adjoint(A, 1, n, x, y)
    assert rc == capi.ERR_ARGUMENT
    assert b"static scratch" in capi.lib().tval3g_last_error()
