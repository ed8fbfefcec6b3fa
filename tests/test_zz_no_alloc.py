"""The allocation-free solve, b2m_dev_MatrixLinEQSolveNoAlloc, against the allocating entry point
and the oracle.

It serves callers that may not allocate device memory -- a host program whose memory manager owns
every device allocation, or a real-time loop with a fixed memory budget.  Its scratch is one static
device array shared by all calls, so the test makes two calls in a row (the second at the maximum
size) to check that nothing from the first call leaks into the second, compares each with
b2m_dev_MatrixLinEQSolve through the C ABI and with the oracle's MatrixLinEQSolve restatement,
and checks that a singular system is reported through the device result word.
This file is collected last so a run that stops at the first failure has run every other test.
"""
import numpy as np
import pytest

import oracle
from mrmath_b200 import _lib, inputs, linalg as L

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # same bar as the other solve parity tests


def _noalloc(stream, A, B, X, status):
    return _lib.lib.b2m_dev_MatrixLinEQSolveNoAlloc(
        stream, A.data_ptr(), A.stride(0) * 8, A.shape[1], B.data_ptr(), B.stride(0) * 8, X.data_ptr(),
        X.stride(0) * 8, B.shape[1], status.data_ptr() if status is not None else None)


def test_noalloc_solve_matches_allocating_solve_twice(ctx):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    for n, k, seed in ((300, 5, 1), (512, 64, 2)):
        r = inputs.rng(seed)
        # R - 0.5 + 2 sqrt(n) I has ||R - 0.5||_2 ~ 0.58 sqrt(n), so kappa < 2: two correct solves
        # then agree to a few ulps, which is what the 1e-12 bar against the oracle can hold
        a_np, b_np = r.random_sample((n, n)) - 0.5 + 2.0 * np.sqrt(n) * np.eye(n), r.standard_normal((n, k))
        a, b = torch.from_numpy(a_np).cuda(), torch.from_numpy(b_np).cuda()
        x_ref = torch.empty_like(b)
        st_ref = torch.zeros(1, dtype=torch.int32, device="cuda")
        L.dev_MatrixLinEQSolve(a, b, x_ref, status=st_ref, ctx=ctx)
        x = torch.full_like(b, float("nan"))
        st = torch.full((1,), 7, dtype=torch.int32, device="cuda")
        assert _noalloc(stream, a, b, x, st) == _lib.OK
        torch.cuda.synchronize()
        assert int(st.item()) == 0 and int(st_ref.item()) == 0
        xg = x.cpu().numpy()
        xr = x_ref.cpu().numpy()
        assert np.linalg.norm(xg - xr) <= RTOL * np.linalg.norm(xr)
        rc, xo = oracle.lineq_solve(a_np, b_np, row_quirk=False)
        assert rc == 0 and np.linalg.norm(xg - xo) <= RTOL * np.linalg.norm(xo)


def test_noalloc_reports_singular(ctx):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    a = torch.eye(50, dtype=torch.float64, device="cuda")
    a[:, 17] = 0.0
    b = torch.ones(50, 2, dtype=torch.float64, device="cuda")
    x = torch.empty_like(b)
    st = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    assert _noalloc(stream, a, b, x, st) == _lib.OK
    torch.cuda.synchronize()
    assert int(st.item()) == _lib.SINGULAR
    # the next call on the shared scratch starts clean
    a2 = torch.eye(50, dtype=torch.float64, device="cuda") * 2.0
    assert _noalloc(stream, a2, b, x, st) == _lib.OK
    torch.cuda.synchronize()
    assert int(st.item()) == 0 and torch.equal(x, b / 2.0)


def test_noalloc_rejects_sizes_beyond_its_scratch(ctx):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    a = torch.eye(513, dtype=torch.float64, device="cuda")
    b = torch.ones(513, 1, dtype=torch.float64, device="cuda")
    x = torch.empty_like(b)
    assert _noalloc(stream, a, b, x, None) == _lib.ERR_UNSUPPORTED
    a = torch.eye(8, dtype=torch.float64, device="cuda")
    b = torch.ones(8, 65, dtype=torch.float64, device="cuda")
    x = torch.empty_like(b)
    assert _noalloc(stream, a, b, x, None) == _lib.ERR_UNSUPPORTED
