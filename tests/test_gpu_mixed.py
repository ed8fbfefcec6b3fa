"""Mixed-precision solve: FP32 tcgen05 factorisation + FP64 refinement must reach the FP64
backward-error target n * 2^-53 (residual checked with the oracle's compensated Dot2)."""
import numpy as np
import pytest

import oracle
from mrmath_b200 import _lib, inputs, linalg as L

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,k", [(64, 1), (300, 3), (1000, 16), (2048, 16)])
@pytest.mark.parametrize("mode", [_lib.MIXED_TF32, _lib.MIXED_3XTF32])
def test_mixed_solve_reaches_fp64_backward_error(ctx, n, k, mode):
    r = inputs.rng(100 + n)
    a = r.random_sample((n, n)) - 0.5
    a[np.diag_indices(n)] += 2.0
    b = r.standard_normal((n, k))
    st, x, rep = L.MatrixLinEQSolveMixed(a, b, mode=mode, ctx=ctx)
    assert st == 0
    bound = n * 2.0 ** -53
    eta = oracle.backward_error(a, x, b)
    assert eta <= bound, (eta, rep)
    assert rep["iterations"] >= 1 and rep["backward_error"] <= bound
    if mode == _lib.MIXED_3XTF32:  # 3xTF32 converges without the FP64 fallback on these systems
        assert rep["fell_back"] == 0


@pytest.mark.parametrize("n,k", [(257, 2), (513, 5), (4100, 16), (8500, 4)])
def test_mixed_solve_ragged_and_tall(ctx, n, k):
    """Ragged leaves and outer panels (n not a multiple of 32 / 256) and, at n = 8500, a
    tournament tree with two merge levels (17 chunks of 512 rows)."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(n)
    A = torch.rand((n, n), generator=g, device="cuda", dtype=torch.float64) - 0.5
    A += torch.eye(n, device="cuda", dtype=torch.float64) * 2.0
    B = torch.randn((n, k), generator=g, device="cuda", dtype=torch.float64)
    X = torch.empty_like(B)
    st, rep = L.dev_MatrixLinEQSolveMixed(A, B, X, mode=_lib.MIXED_3XTF32, ctx=ctx)
    torch.cuda.synchronize()
    assert st == 0 and rep["fell_back"] == 0, rep
    a, b, x = A.cpu().numpy(), B.cpu().numpy(), X.cpu().numpy()
    eta = oracle.backward_error(a, x, b)
    assert eta <= n * 2.0 ** -53, (eta, rep)


@pytest.mark.parametrize("kappa", [1e2, 1e4, 1e5])
def test_mixed_solve_kappa_family(ctx, kappa):
    """The benchmark's construction A = U diag(s) V^T at n = 1024."""
    import torch
    A, B = inputs.c2_kappa(1024, kappa, 16, seed=7, device="cuda")
    a, b = A.cpu().numpy(), B.cpu().numpy()
    st, x, rep = L.MatrixLinEQSolveMixed(a, b, mode=_lib.MIXED_3XTF32, ctx=ctx)
    assert st == 0
    eta = oracle.backward_error(a, x, b)
    assert eta <= 1024 * 2.0 ** -53, (eta, rep)
    # TF32 alone may need the FP64 fallback at kappa = 1e5; the answer must still meet the bound
    st, x1, rep1 = L.MatrixLinEQSolveMixed(a, b, mode=_lib.MIXED_TF32, ctx=ctx)
    assert st == 0 and oracle.backward_error(a, x1, b) <= 1024 * 2.0 ** -53, rep1


def test_mixed_device_api_and_singular(ctx):
    import torch
    r = inputs.rng(3)
    n = 512
    a = r.random_sample((n, n)) + n * np.eye(n)
    b = r.standard_normal((n, 4))
    A = torch.from_numpy(a).cuda()
    B = torch.from_numpy(b).cuda()
    X = torch.empty_like(B)
    st, rep = L.dev_MatrixLinEQSolveMixed(A, B, X, ctx=ctx)
    torch.cuda.synchronize()
    assert st == 0 and rep["fell_back"] == 0
    assert oracle.backward_error(a, X.cpu().numpy(), b) <= n * 2.0 ** -53
    z = np.eye(40)
    z[:, 7] = 0.0
    st, _, rep = L.MatrixLinEQSolveMixed(z, np.ones((40, 1)), ctx=ctx)
    assert st == 1
