"""Adjoint of the LU solve (b2m_MatrixLinEQSolveAdjoint and its device twin, wrapped by
mrmath_b200.autograd for gradient checking).

The reference has no adjoint; the gradient of loss = w^T A^-1 b is checked two ways:
  * against the closed form built from the reference's own solves (the oracle's
    MatrixLinEQSolve restatement): db = A^-T w, dA = -db x^T;
  * against central finite differences, h = 1e-6, on 64 random entries of A.  A perturbation of
    1e-6 moves the loss by ~1e-11 of its size, so each perturbed loss is evaluated to ~u^2: x0 from
    the GPU solve, one correction d from a Dot2 residual kept separate, and w^T x0 summed exactly.
"""
from fractions import Fraction

import numpy as np
import pytest

import oracle
from mrmath_b200 import inputs, linalg as L

pytestmark = pytest.mark.gpu

REL = 1e-12  # closed form vs adjoint kernel (both FP64 solves of a well-conditioned system)
FD_REL = 1e-6  # finite differences, per entry


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("n,k", [(200, 1), (333, 3), (1000, 16), (700, 40)])
def test_adjoint_matches_closed_form(ctx, n, k):
    r = inputs.rng(500 + n)
    a = r.random_sample((n, n)) * 2.0 - 1.0
    # ||R||_2 ~ 1.15 sqrt(n) for R uniform on (-1, 1): + 2 sqrt(n) I keeps kappa below ~4, so two
    # correct FP64 solves agree to a few ulps and the 1e-12 bar holds for the products below
    a[np.diag_indices(n)] += 2.0 * np.sqrt(n)
    b = r.standard_normal((n, k))
    g = r.standard_normal((n, k))
    st, lu, indx = L.MatrixLUDecomp(a, ctx=ctx)
    assert st == 0
    x = b.copy()
    L.MatrixLUBackSubst(lu, indx, x, ctx=ctx)
    dA = np.empty((n, n))
    lam = L.MatrixLinEQSolveAdjoint(lu, indx, x, g, dA=dA, ctx=ctx)
    rc, x_ref = oracle.lineq_solve(a, b)
    rc2, lam_ref = oracle.lineq_solve(np.ascontiguousarray(a.T), g)
    assert rc == 0 and rc2 == 0
    assert _rel(lam, lam_ref) < REL
    assert _rel(dA, -lam_ref @ x_ref.T) < REL
    # op = DO_ADD accumulates, dA = None skips the update
    acc = np.ones((n, n))
    L.MatrixLinEQSolveAdjoint(lu, indx, x, g, dA=acc, op=L.DO_ADD, ctx=ctx)
    assert _rel(acc, 1.0 - lam_ref @ x_ref.T) < REL
    lam2 = L.MatrixLinEQSolveAdjoint(lu, indx, x, g, dA=None, ctx=ctx)
    assert np.array_equal(lam, lam2)


def test_adjoint_device_twin_and_strides(ctx):
    import torch
    n, k = 513, 5
    r = inputs.rng(77)
    a = r.random_sample((n, n)) + n * np.eye(n)
    g = r.standard_normal((n, k))
    b = r.standard_normal((n, k))
    A = torch.from_numpy(a).cuda()
    LU = torch.empty((n, n + 3), dtype=torch.float64, device="cuda")[:, :n]  # padded rows
    LU.copy_(A)
    indx = torch.zeros(n, dtype=torch.int32, device="cuda")
    L.dev_MatrixLUDecompInPlace(LU, indx, ctx=ctx)
    X = torch.from_numpy(b).cuda()
    L.dev_MatrixLUBackSubst(LU, indx, X, ctx=ctx)
    G = torch.from_numpy(g).cuda()
    Lam = torch.empty((n, k + 1), dtype=torch.float64, device="cuda")[:, :k]
    dA = torch.empty((n, n), dtype=torch.float64, device="cuda")
    L.dev_MatrixLinEQSolveAdjoint(LU, indx, X, G, Lam, dA, ctx=ctx)
    torch.cuda.synchronize()
    lam_ref = np.linalg.solve(a.T, g)
    x_ref = np.linalg.solve(a, b)
    assert _rel(Lam.cpu().numpy(), lam_ref) < 1e-12
    assert _rel(dA.cpu().numpy(), -lam_ref @ x_ref.T) < 1e-12


def _exact_dot(w, x):
    return sum((Fraction(float(wi)) * Fraction(float(xi)) for wi, xi in zip(w, x)), Fraction(0))


def test_adjoint_gradient_c4_finite_differences(ctx):
    """loss = w^T A^-1 b, n = 4096, A = R + 4096 I with R uniform [-1, 1), b and w Gaussian."""
    import torch

    from mrmath_b200 import autograd

    n = 4096
    r = inputs.rng(4096)
    a = r.random_sample((n, n)) * 2.0 - 1.0 + n * np.eye(n)
    b = r.standard_normal(n)
    w = r.standard_normal(n)
    At = torch.from_numpy(a).cuda().requires_grad_(True)
    bt = torch.from_numpy(b).cuda().requires_grad_(True)
    wt = torch.from_numpy(w).cuda()
    x = autograd.solve(At, bt, ctx)
    loss = torch.dot(wt, x)
    loss.backward()
    gA = At.grad.cpu().numpy()
    gb = bt.grad.cpu().numpy()

    # closed form from the reference algorithm's own (threaded) solves
    oracle.set_num_threads(8)
    rc, x_ref = oracle.thr_lineq_solve(a, b.reshape(n, 1))
    rc2, lam_ref = oracle.thr_lineq_solve(np.ascontiguousarray(a.T), w.reshape(n, 1))
    assert rc == 0 and rc2 == 0
    assert _rel(gb, lam_ref[:, 0]) < REL
    idx = r.randint(0, n, size=(64, 2))
    closed = np.array([-lam_ref[i, 0] * x_ref[j, 0] for i, j in idx])
    assert _rel(np.array([gA[i, j] for i, j in idx]), closed) < REL

    # central finite differences, h = 1e-6, each loss to ~u^2
    Ad = torch.from_numpy(a).cuda()
    Bd = torch.from_numpy(b.reshape(n, 1)).cuda()
    Xd = torch.empty_like(Bd)
    Dd = torch.empty_like(Bd)
    h = 1e-6

    def loss_at():
        L.dev_MatrixLinEQSolve(Ad, Bd, Xd, ctx=ctx)
        x0 = Xd.cpu().numpy()
        res = oracle.residual_dot2(a, x0, b.reshape(n, 1))
        L.dev_MatrixLinEQSolve(Ad, torch.from_numpy(res).cuda(), Dd, ctx=ctx)
        return _exact_dot(w, x0[:, 0]) + Fraction(float(np.dot(w, Dd.cpu().numpy()[:, 0])))

    worst = 0.0
    for i, j in idx:
        aij = a[i, j]
        vals = []
        for s in (1.0, -1.0):
            v = aij + s * h
            a[i, j] = v
            Ad[i, j] = v
            vals.append((loss_at(), v))
        a[i, j] = aij
        Ad[i, j] = aij
        (lp, vp), (lm, vm) = vals
        fd = float((lp - lm) / (Fraction(vp) - Fraction(vm)))
        worst = max(worst, abs(fd - gA[i, j]) / abs(fd))
    assert worst < FD_REL, worst
