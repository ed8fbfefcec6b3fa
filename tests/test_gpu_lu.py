"""Parity of the CUDA plain-FP64 path (through the C ABI) with the oracle restatement.

Bar (north star): pivot vectors bit-exact; LU factors and solutions within 1e-12 relative in the
Frobenius norm; the reference's 2x2 known answers bitwise.
"""
import numpy as np
import pytest

import oracle
from mrmath_b200 import linalg as L

pytestmark = pytest.mark.gpu

FACTOR_RTOL = 1e-12   # ||LU_gpu - LU_oracle||_F / ||LU_oracle||_F


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_lu_kat_2x2_bitwise(ctx):
    A = np.array([[1.0, 2.0], [2.0, -1.0]])
    st, idx = L.MatrixLUDecompInPlace(A, ctx=ctx)
    assert st == 0 and list(idx) == [1, 1]
    assert A.tobytes() == np.array([[2.0, -1.0], [0.5, 2.5]]).tobytes()
    B = np.array([[2.0], [-1.0]])
    L.MatrixLUBackSubst(A, idx, B, ctx=ctx)
    assert B.tobytes() == np.array([[0.0], [1.0]]).tobytes()


def test_lu_kat_strided(ctx):
    buf = np.array([[1.0, 2.0, 0.0], [2.0, -1.0, 0.0]])
    st, idx = L.MatrixLUDecompInPlace(buf[:, :2], ctx=ctx)
    assert st == 0 and buf.tobytes() == np.array([[2.0, -1.0, 0.0], [0.5, 2.5, 0.0]]).tobytes()
    Bb = np.array([[2.0, 0.0], [-1.0, 0.0]])
    L.MatrixLUBackSubst(buf[:, :2], idx, Bb[:, :1], ctx=ctx)
    assert Bb.tobytes() == np.array([[0.0, 0.0], [1.0, 0.0]]).tobytes()


def test_inverse_det_singular_kats(ctx):
    inv = np.array([[1.0, 2.0], [2.0, -1.0]])
    assert L.MatrixInverseInPlace(inv, ctx=ctx) == 0
    assert inv.tobytes() == np.array([[0.2, 0.4], [0.4, -0.2]]).tobytes()
    s = np.array([[1.0, 2, 3], [2, 4, 6], [3, 3, -1]])
    s0 = s.copy()
    assert L.MatrixInverseInPlace(s, ctx=ctx) == 1
    assert np.array_equal(s, s0)  # left untouched on failure
    assert L.MatrixDeterminant(np.array([[1.0, 2.0], [2.0, -1.0]]), ctx=ctx) == -5.0
    assert L.MatrixDeterminant(s0, ctx=ctx) == 0.0


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 31, 32, 33, 47, 48, 49, 63, 64, 65, 100, 127, 129, 255, 257, 500, 512, 513, 544, 1000, 1024, 1056, 2048])
def test_lu_odd_sizes(ctx, n):
    r = oracle.Mersenne(seed=1000 + n)
    a = r.uniform(n, n) - 0.5
    ref = a.copy()
    rc0, i0 = oracle.lu_decomp_inplace(ref)
    st, LU, idx = L.MatrixLUDecomp(a, ctx=ctx)
    assert st == rc0 == 0
    assert np.array_equal(idx, i0), f"pivots differ at {np.nonzero(idx != i0)[0][:5]}"
    assert rel(LU, ref) <= FACTOR_RTOL


def test_lu_c1_uniform_1024(ctx):
    """Config: n = 1024, A uniform [0,1) from MT19937 seed 15 (TDoubleMatrix.CreateRand), b continuing."""
    r = oracle.Mersenne(seed=15)
    a = r.uniform(1024, 1024)
    b = r.uniform(1024, 1)
    ref = a.copy()
    rc0, i0 = oracle.lu_decomp_inplace(ref)
    st, LU, idx = L.MatrixLUDecomp(a, ctx=ctx)
    assert st == rc0 == 0
    assert np.array_equal(idx, i0)
    assert rel(LU, ref) <= FACTOR_RTOL
    _, x_ref = oracle.lineq_solve(a, b)
    st, x = L.MatrixLinEQSolve(a, b, ctx=ctx)
    assert st == 0
    assert rel(x, x_ref) <= 1e-12
    assert oracle.backward_error(a, x, b) <= 1024 * 2.0 ** -53


def test_padded_strides_and_multi_rhs(ctx):
    r = oracle.Mersenne(seed=21)
    n, k = 77, 5
    abuf = r.uniform(n, n + 3) - 0.5
    bbuf = r.uniform(n, k + 1) - 0.5
    a = abuf[:, :n]
    b = bbuf[:, :k]
    st, x = L.MatrixLinEQSolve(a, b, ctx=ctx)
    assert st == 0
    _, x_ref = oracle.lineq_solve(np.ascontiguousarray(a), np.ascontiguousarray(b), row_quirk=False)
    assert rel(x, x_ref) <= 1e-12
    # in-place LU on the padded view leaves the padding alone
    pad = abuf[:, n:].copy()
    st, idx = L.MatrixLUDecompInPlace(a, ctx=ctx)
    assert st == 0 and np.array_equal(abuf[:, n:], pad)


@pytest.mark.parametrize("n,k", [(300, 1), (257, 3)])
def test_refinement_steps(ctx, n, k):
    """NumRefinements in {0, 1, 3} against the oracle's MatrixLinEQSolve refinement
    (LinAlgLU.pas:542-586) with each column's residual read along its own column."""
    r = oracle.Mersenne(seed=5 + n)
    a = r.uniform(n, n) - 0.5
    b = r.uniform(n, k) - 0.5
    for nref in (0, 1, 3):
        st, x = L.MatrixLinEQSolve(a, b, num_refinements=nref, ctx=ctx)
        assert st == 0
        rc, x_ref = oracle.lineq_solve(a, b, num_refinements=nref, row_quirk=False)
        assert rc == 0
        assert rel(x, x_ref) <= 1e-12, (nref, rel(x, x_ref))
        assert oracle.backward_error(a, x, b) <= n * 2.0 ** -53


def test_inverse_and_determinant_parity(ctx):
    r = oracle.Mersenne(seed=15)
    a = r.uniform(512, 512) - 0.5
    x = a.copy()
    assert L.MatrixInverseInPlace(x, ctx=ctx) == 0
    y = a.copy()
    assert oracle.inverse_inplace(y) == 0
    assert rel(x, y) <= FACTOR_RTOL, rel(x, y)
    assert np.abs(a @ x - np.eye(512)).max() <= 1e-9
    d = r.uniform(256, 256) / 3.8 - 0.5 / 3.8
    det, det_ref = L.MatrixDeterminant(d, ctx=ctx), oracle.determinant(d)
    assert det != 0 and abs(det - det_ref) <= abs(det_ref) * 1e-10  # TestDeterminant2 tolerance


def test_singular_cases(ctx):
    z = np.eye(6)
    z[:, 3] = 0.0
    st, _ = L.MatrixLUDecompInPlace(z.copy(), ctx=ctx)
    assert st == 1
    st, _ = L.MatrixLinEQSolve(z, np.ones((6, 1)), ctx=ctx)
    assert st == 1
    st, _ = L.MatrixLUDecompInPlace(np.zeros((40, 40)), ctx=ctx)
    assert st == 1
    # a later singular column (rank deficient 100 x 100)
    r = oracle.Mersenne(seed=9)
    a = r.uniform(100, 60) @ r.uniform(60, 100)
    rc0, _ = oracle.lu_decomp_inplace(a.copy())
    st, _ = L.MatrixLUDecompInPlace(a.copy(), ctx=ctx)
    assert st == rc0


@pytest.mark.parametrize("trans", [0, 1, 2])
@pytest.mark.parametrize("op", [0, 1, 2])
def test_gemm_parity(ctx, trans, op):
    r = oracle.Mersenne(seed=31 + 3 * trans + op)
    for (m, n, k) in ((1, 1, 1), (17, 33, 5), (130, 129, 257), (256, 128, 64), (300, 200, 1000)):
        if trans == 0:
            a, b = r.uniform(m, k) - 0.5, r.uniform(k, n) - 0.5
            ref_prod = a @ b
        elif trans == 1:
            a, b = r.uniform(k, m) - 0.5, r.uniform(k, n) - 0.5
            ref_prod = a.T @ b
        else:
            a, b = r.uniform(m, k) - 0.5, r.uniform(n, k) - 0.5
            ref_prod = a @ b.T
        c0 = r.uniform(m, n)
        c = c0.copy()
        L.MatrixMultEx(c, a, b, op=op, trans=trans, ctx=ctx)
        ref = oracle_c = c0.copy()
        oracle.block_mult(oracle_c, a, b, block=128, op=op, trans=trans)
        tol = 4 * k * 2.0 ** -53 * (np.abs(a).max() * np.abs(b).max() * k + 1.0)
        assert np.abs(c - ref).max() <= tol, (m, n, k)
        expect = {0: ref_prod, 1: c0 + ref_prod, 2: c0 - ref_prod}[op]
        assert np.abs(c - expect).max() <= tol


def test_device_api_torch(ctx):
    import torch
    r = oracle.Mersenne(seed=44)
    n, k = 640, 16
    a = r.uniform(n, n) - 0.5
    b = r.uniform(n, k) - 0.5
    A = torch.from_numpy(a).cuda()
    B = torch.from_numpy(b).cuda()
    X = torch.empty_like(B)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.dev_MatrixLinEQSolve(A, B, X, status=status, ctx=ctx)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    _, x_ref = oracle.lineq_solve(a, b, row_quirk=False)
    assert rel(X.cpu().numpy(), x_ref) <= 1e-12
    LU = A.clone()
    idx = torch.zeros(n, dtype=torch.int32, device="cuda")
    L.dev_MatrixLUDecompInPlace(LU, idx, status=status, ctx=ctx)
    torch.cuda.synchronize()
    ref = a.copy()
    _, i0 = oracle.lu_decomp_inplace(ref)
    assert np.array_equal(idx.cpu().numpy(), i0)
    assert rel(LU.cpu().numpy(), ref) <= FACTOR_RTOL
    Y = B.clone()
    L.dev_MatrixLUBackSubst(LU, idx, Y, ctx=ctx)
    torch.cuda.synchronize()
    assert rel(Y.cpu().numpy(), x_ref) <= 1e-12
    C = torch.empty(n, k, dtype=torch.float64, device="cuda")
    L.dev_MatrixMultEx(C, A, B, ctx=ctx)
    torch.cuda.synchronize()
    np.testing.assert_allclose(C.cpu().numpy(), a @ b, rtol=0, atol=1e-12)
