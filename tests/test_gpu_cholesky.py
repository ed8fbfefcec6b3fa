"""Cholesky factorisation and solve (LinAlgCholesky.pas) through the C ABI against the oracle's
restatement of MatrixCholeskyInPlace4 / MatrixCholeskyInPlace / MatrixCholeskySolveLinEq.

Bar: the reference's 3 x 3 known answers (TestLineEquations.pas:494-524); factors and solutions
within 1e-12 relative (Frobenius) of the oracle's; the strict upper triangle (and, for the
Numerical-Recipes form, the diagonal) never written; crNoPositiveDefinite on the same inputs."""
import numpy as np
import pytest

import oracle
from mrmath_b200 import linalg as L

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def spd(n, seed):
    r = oracle.Mersenne(seed=seed)
    g = r.uniform(n, n) - 0.5
    a = oracle.matrix_mult(g, np.ascontiguousarray(g.T))
    a[np.diag_indices(n)] += 0.25 * n
    return a


def test_cholesky_kat_3x3(ctx):
    A = np.array([[1.0, 2, 2], [-1, 4, -2], [2, 2, -1]])
    X = oracle.matrix_mult(A, np.ascontiguousarray(A.T))
    x = X.copy()
    P = np.zeros((3, 4))  # LineWidthP = 4 doubles, as the reference's test passes it
    assert L.MatrixCholeskyInPlace(x, P, ctx=ctx) == 0
    xo, Po = X.copy(), np.zeros((3, 4))
    assert oracle.cholesky_nr(xo, Po) == 0
    assert rel(np.tril(x, -1), np.tril(xo, -1)) <= RTOL and rel(P[:, 0], Po[:, 0]) <= RTOL
    assert np.array_equal(np.triu(x), np.triu(X))  # diagonal and upper triangle untouched
    B = np.array([[2.0], [-1.0], [-1.0]])
    res = L.MatrixCholeskySolveLinEq(x, B, P, ctx=ctx)
    np.testing.assert_allclose(res.ravel(), [0.338888889, 0.00555555556, -0.2666666667], atol=1e-9)
    assert rel(res, oracle.cholesky_solve_nr(xo, Po, B)) <= RTOL
    # A itself is not positive definite: crNoPositiveDefinite, A unchanged
    a = A.copy()
    assert L.MatrixCholeskyInPlace(a, np.zeros((3, 4)), ctx=ctx) == 1 and np.array_equal(a, A)
    a = A.copy()
    assert L.MatrixCholeskyInPlace4(a, ctx=ctx) == 1 and np.array_equal(a, A)


@pytest.mark.parametrize("n", [1, 2, 3, 31, 32, 33, 100, 255, 256, 257, 511, 1000, 2048])
def test_cholesky_inplace4_matches_oracle(ctx, n):
    a = spd(n, 50 + n)
    a0 = a.copy()
    ref = a.copy()
    assert oracle.cholesky_inplace4(ref) == 0
    assert L.MatrixCholeskyInPlace4(a, ctx=ctx) == 0
    assert rel(np.tril(a), np.tril(ref)) <= RTOL, rel(np.tril(a), np.tril(ref))
    assert np.array_equal(np.triu(a, 1), np.triu(a0, 1))
    # solve with the InPlace4 form (diagonal in A) for several right-hand sides
    b = oracle.Mersenne(seed=n).uniform(n, 5) - 0.5
    x = L.MatrixCholeskySolveLinEq(a, b, ctx=ctx)
    _, x_lu = oracle.lineq_solve(a0, b, row_quirk=False)
    assert rel(x, x_lu) <= RTOL
    assert oracle.backward_error(a0, x, b) <= max(n, 4) * 2.0 ** -53


def test_cholesky_padded_strides_and_nr_form(ctx):
    n = 300
    a = spd(n, 9)
    buf = np.full((n, n + 5), 7.0)
    buf[:, :n] = a
    view = buf[:, :n]
    P = np.zeros((n, 3))
    assert L.MatrixCholeskyInPlace(view, P, ctx=ctx) == 0
    ref, Pr = a.copy(), np.zeros((n, 1))
    assert oracle.cholesky_nr(ref, Pr) == 0
    assert rel(np.tril(view, -1), np.tril(ref, -1)) <= RTOL and rel(P[:, 0], Pr[:, 0]) <= RTOL
    assert np.array_equal(np.triu(view), np.triu(a)) and np.all(buf[:, n:] == 7.0)
    b = oracle.Mersenne(seed=4).uniform(n, 1) - 0.5
    x = L.MatrixCholeskySolveLinEq(view, b, P, ctx=ctx)
    assert rel(x, oracle.cholesky_solve_nr(ref, Pr, b)) <= RTOL


def test_cholesky_not_positive_definite_later_column(ctx):
    n = 200
    a = spd(n, 11)
    a[150, 150] = -1e6  # fails at column 150, after 4 full leaves and an outer panel
    ref = a.copy()
    assert oracle.cholesky_inplace4(ref) == 1
    b = a.copy()
    assert L.MatrixCholeskyInPlace4(b, ctx=ctx) == 1 and np.array_equal(b, a)
    a[0, 0] = np.nan
    assert oracle.cholesky_inplace4(a.copy()) == 1 and L.MatrixCholeskyInPlace4(a.copy(), ctx=ctx) == 1


def test_cholesky_device_twins_8192(ctx):
    import torch
    n = 8192
    a = spd(n, 8192)
    A = torch.from_numpy(a).cuda()
    F = A.clone()
    status = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    L.dev_MatrixCholeskyInPlace4(F, status=status, ctx=ctx)
    b = oracle.Mersenne(seed=3).uniform(n, 16) - 0.5
    B = torch.from_numpy(b).cuda()
    X = torch.empty_like(B)
    L.dev_MatrixCholeskySolveLinEq(F, B, X, ctx=ctx)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    assert torch.equal(torch.triu(F, 1), torch.triu(A, 1))
    assert oracle.backward_error(a, X.cpu().numpy(), b) <= n * 2.0 ** -53
    # the factor reproduces A: ||L L^T - A|| within the Cholesky backward-error bound
    Lf = torch.tril(F)
    err = float(((Lf @ Lf.T - A).abs().max() / A.abs().max()).item())
    assert err <= n * 2.0 ** -53, err
