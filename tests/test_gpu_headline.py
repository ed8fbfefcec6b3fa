"""Parity at the benchmarked sizes, through the C ABI, against the oracle.

* The mixed-precision solve on the benchmark's own system (n = 8192, 16 right-hand sides,
  A = U diag(s) V^T with kappa in {1e2, 1e4, 1e5}): the oracle's compensated (Dot2) backward error
  must be <= n 2^-53 without the FP64 fallback (3xTF32), and the plain FP64 drop-in on the same
  system must meet the same bound.
* The plain FP64 LU (MatrixLUDecomp's drop-in) at n = 8192 (16-CTA cluster panel, 32-column
  leaves) and n = 9000 (16-column leaves): pivots bit-exact against the oracle's restatement of the
  reference's threaded LU (ThrMatrixLUDecomp, LinAlgLU.pas:674-803), factors within
  max(1e-12, n 2^-53) relative (Frobenius).  The pivots do not depend on the summation order of the
  Schur updates, the factors do at the rounding level, and that difference grows with n (1.5e-12
  at n = 16500), so the bar above n = 9000 is n 2^-53.
"""
import numpy as np
import pytest

import oracle
from mrmath_b200 import _lib, inputs, linalg as L

pytestmark = pytest.mark.gpu

N = 8192


@pytest.mark.parametrize("kappa", [1e2, 1e4, 1e5])
def test_headline_system_mixed_and_plain(ctx, kappa):
    import torch
    A, B = inputs.c2_kappa(N, kappa, 16, seed=15, device="cuda")
    X = torch.empty_like(B)
    st, rep = L.dev_MatrixLinEQSolveMixed(A, B, X, mode=_lib.MIXED_3XTF32, ctx=ctx)
    torch.cuda.synchronize()
    assert st == 0 and rep["fell_back"] == 0, rep
    a, b, x = A.cpu().numpy(), B.cpu().numpy(), X.cpu().numpy()
    bound = N * 2.0 ** -53
    eta = oracle.backward_error(a, x, b)
    assert eta <= bound, (kappa, eta, rep)
    # the library's own FP64 residual agrees with the compensated one to within its rounding
    assert rep["backward_error"] <= bound and abs(rep["backward_error"] - eta) <= 0.1 * bound, (eta, rep)
    # the forward-error estimate (last correction scaled by the observed contraction) lies below
    # FP32 accuracy and within an order of magnitude of the a-priori kappa * eta scale
    assert 0.0 < rep["forward_error"] <= 10 * kappa * bound and rep["forward_error"] < 1e-7, rep
    # the plain FP64 drop-in on the same system
    Xp = torch.empty_like(B)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.dev_MatrixLinEQSolve(A, B, Xp, status=status, ctx=ctx)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    xp = Xp.cpu().numpy()
    assert oracle.backward_error(a, xp, b) <= bound
    # two backward-stable solutions of the same system differ by about kappa times their errors
    diff = np.max(np.abs(x - xp)) / np.max(np.abs(xp))
    assert diff <= kappa * 4 * bound, (kappa, diff)


@pytest.mark.parametrize("n", [8192, 9000, 16500])
def test_plain_lu_pivots_at_bench_sizes(ctx, n):
    """32-column leaves (n <= 8192), 16-column leaves (n <= 16384) and 8-column leaves on
    16-CTA clusters holding up to 32768 panel rows (n = 16500)."""
    r = oracle.Mersenne(seed=2 * n + 1)
    a = r.uniform(n, n) - 0.5
    ref = a.copy()
    rc0, i0 = oracle.thr_lu_decomp_inplace(ref)
    assert rc0 == 0
    st, lu, idx = L.MatrixLUDecomp(a, ctx=ctx)
    assert st == 0
    bad = np.nonzero(idx != i0)[0]
    assert bad.size == 0, f"pivots differ at {bad[:5]} (n={n})"
    err = np.linalg.norm(lu - ref) / np.linalg.norm(ref)
    assert err <= max(1e-12, n * 2.0 ** -53), (n, err)


def test_plain_solve_20000(ctx):
    """MatrixLinEQSolve's drop-in beyond n = 16384 (8-column leaves, short-K Schur updates),
    checked by the oracle's compensated backward error (the oracle's own LU at this order would
    take minutes on the host)."""
    import torch
    n = 20000
    r = inputs.rng(20000)
    a = r.random_sample((n, n)) - 0.5
    b = r.standard_normal((n, 2))
    A, B = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    X = torch.empty_like(B)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.dev_MatrixLinEQSolve(A, B, X, status=status, ctx=ctx)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    x = X.cpu().numpy()
    assert np.all(np.isfinite(x))
    assert oracle.backward_error(a, x, b) <= n * 2.0 ** -53
