"""The oracle against the reference's own known answers (CPU only).

Pins: Test/marsenneTwistOrig.txt byte for byte (TestRandom.pas:249-311); the LU, back-substitution,
inverse, singularity and determinant known answers of Test/TestLineEquations.pas; the GEMM known
answers of Test/TestSimpleMatrixOperations.pas:1712-1727, Test/TestFMA.pas:415-449 and
Test/TestMatrixClass.pas:473-509; and the reference's own differential tests (single-threaded vs
threaded LU / inverse / determinant / solve, TestLineEquations.pas:121-176, 644-678, 725-756, 833-870).
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_mt19937_fixture_byte_for_byte():
    g = json.load(open(os.path.join(GOLDEN, "mt19937ar_kat.json")))
    r = oracle.Mersenne(key=g["init_key"])
    ints = [r.lw(0xFFFFFFFF) for _ in range(1000)]
    assert ints == g["genrand_int32"]
    reals = [r.random() for _ in range(1000)]
    # rebuild the file exactly as TestMersenneTwisterStdTest writes it
    s = "1000 outputs of genrand_int32()\r\n"
    for i in range(200):
        s += "%10u %10u %10u %10u %10u \r\n" % tuple(ints[5 * i:5 * i + 5])
    s += "\r\n1000 outputs of genrand_real2()\r\n"
    for i in range(200):
        s += "%10.8f %10.8f %10.8f %10.8f %10.8f \r\n" % tuple(reals[5 * i:5 * i + 5])
    assert len(s) == g["size"]
    assert hashlib.sha256(s.encode()).hexdigest() == g["sha256"]


def test_lu_decomp_2x2_kat():
    # TestLUDecomp1 TestLineEquations.pas:812-831
    A = np.array([[1.0, 2.0], [2.0, -1.0]])
    rc, idx = oracle.lu_decomp_inplace(A)
    assert rc == 0
    assert A.tobytes() == np.array([[2.0, -1.0], [0.5, 2.5]]).tobytes()
    assert list(idx) == [1, 1]


def test_lu_backsubst_kats():
    # TestLUBackSubst1 :758-782
    A = np.array([[1.0, 2.0], [2.0, -1.0]])
    rc, idx = oracle.lu_decomp_inplace(A)
    B = np.array([[2.0], [-1.0]])
    oracle.lu_backsubst(A, idx, B)
    assert B.tobytes() == np.array([[0.0], [1.0]]).tobytes()
    # TestLUBackSubst2 :784-810: LineWidth 3*8 for A, 2*8 for B
    buf = np.array([[1.0, 2.0, 0.0], [2.0, -1.0, 0.0]])
    rc, idx = oracle.lu_decomp_inplace(buf[:, :2])
    assert rc == 0 and buf.tobytes() == np.array([[2.0, -1.0, 0.0], [0.5, 2.5, 0.0]]).tobytes()
    Bb = np.array([[2.0, 0.0], [-1.0, 0.0]])
    oracle.lu_backsubst(buf[:, :2], idx, Bb[:, :1])
    assert Bb.tobytes() == np.array([[0.0, 0.0], [1.0, 0.0]]).tobytes()


def test_inverse_and_singular_kats():
    # TestInvert1 :702-713 (bitwise), TestInvert2 :715-723 (singular)
    inv = np.array([[1.0, 2.0], [2.0, -1.0]])
    assert oracle.inverse_inplace(inv) == 0
    assert inv.tobytes() == np.array([[0.2, 0.4], [0.4, -0.2]]).tobytes()
    s = np.array([[1.0, 2, 3], [2, 4, 6], [3, 3, -1]])
    assert oracle.inverse_inplace(s) == 1


def test_determinant_kat():
    # TestDeterminant1 :635-642
    assert oracle.determinant(np.array([[1.0, 2.0], [2.0, -1.0]])) == -5.0


def test_gemm_kats():
    # TestSimpleMatrixOperations.TestMult :1712-1727
    mt1 = np.arange(6.0).reshape(2, 3)
    mt2 = np.arange(1.0, 7.0).reshape(3, 2)
    oracle.set_mode("generic")
    c = np.zeros((2, 2))
    oracle.lib.orc_generic_mult(oracle._p(c), 16, oracle._p(mt1), oracle._p(mt2), 3, 2, 2, 3, 24, 16)
    assert c.tobytes() == np.array([[13.0, 16.0], [40.0, 52.0]]).tobytes()
    oracle.set_mode("fma")
    # second case: mt2 + 1 element, LineWidth 3*8, 2x2 blocks
    buf2 = np.arange(1.0, 7.0)
    c2 = np.zeros((2, 2))
    p2 = buf2.ctypes.data + 8
    import ctypes
    oracle.lib.orc_generic_mult(oracle._p(c2), 16, oracle._p(mt1), ctypes.cast(p2, oracle._pd), 2, 2, 2, 2, 24, 24)
    assert c2.tobytes() == np.array([[5.0, 6.0], [26.0, 33.0]]).tobytes()
    # TestFMA.TestFMAMult :415-449 (4x4 padded, 1e-10)
    mt4 = np.array([0, 1, 2, 4, 3, 4, 5, 5, 6, 7, 8, 6, 7, 8, 9, 10.0]).reshape(4, 4)
    mt5 = np.array([-1, 0, 1, 1, 2, 3, 4, 2, 5, 6, 7, 3, 4, 5, 6, 7.0]).reshape(4, 4)
    mt6 = np.array([28, 35, 42, 36, 50, 67, 84, 61, 72, 99, 126, 86, 94, 128, 162, 120.0]).reshape(4, 4)
    np.testing.assert_allclose(oracle.matrix_mult(mt4, mt5), mt6, atol=1e-10)
    # TestTDoubleMatrix.TestMult2 :473-509: line matrices of ones * twos
    for w, h, ref in ((610, 62, 1220.0), (611, 62, 1222.0), (611, 63, 1222.0)):
        a = np.ones((h, w))
        b = np.full((w, 1), 2.0)
        assert np.all(np.abs(oracle.matrix_mult(a, b) - ref) <= 1e-12)


def test_blocked_gemm_matches_generic_and_numpy():
    r = oracle.Mersenne(seed=7)
    for (m, k, n) in ((130, 257, 129), (64, 48, 5), (3, 700, 4), (513, 520, 515)):
        a = r.uniform(m, k) - 0.5
        b = r.uniform(k, n) - 0.5
        c = np.zeros((m, n))
        oracle.block_mult(c, a, b, block=48, op=0)
        ref = a @ b
        assert np.abs(c - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()) * k
        # doSub on top of a copy gives ~0
        d = ref.copy()
        oracle.block_mult(d, a, b, block=48, op=2)
        assert np.abs(d).max() <= 1e-11 * k
    # T1 / T2 variants
    a = r.uniform(100, 70)
    b = r.uniform(100, 90)
    c = np.zeros((70, 90))
    oracle.block_mult(c, a, b, block=32, op=0, trans=1)
    np.testing.assert_allclose(c, a.T @ b, rtol=1e-13, atol=1e-12)
    b2 = r.uniform(90, 70)
    c2 = np.zeros((100, 90))
    oracle.block_mult(c2, a, b2, block=32, op=0, trans=2)
    np.testing.assert_allclose(c2, a @ b2.T, rtol=1e-13, atol=1e-12)


def test_reference_differential_lu_threaded_vs_single():
    # TestBigLUDecomp :121-176 uses RandSeed 15 + Random - 0.5 (the FPC/Delphi system RNG, not in the
    # reference tree); the same test body runs here on MT19937 seed 15 inputs.
    r = oracle.Mersenne(seed=15)
    x = r.uniform(1024, 1024) - 0.5
    y = x.copy()
    rc1, i1 = oracle.lu_decomp_inplace(x)
    rc2, i2 = oracle.thr_lu_decomp_inplace(y)
    assert rc1 == rc2 == 0
    assert np.array_equal(i1, i2)
    assert np.abs(x - y).max() <= 1e-4   # CheckMtxIdx default epsilon
    assert oracle.min_pivot_gap(r.uniform(64, 64)) > 0.0


def test_reference_differential_inverse_det_solve():
    r = oracle.Mersenne(seed=15)
    a = r.uniform(512, 512) - 0.5
    x = a.copy()
    y = a.copy()
    assert oracle.inverse_inplace(x) == 0 and oracle.thr_inverse_inplace(y) == 0
    assert np.abs(x - y).max() <= 1e-4
    d = r.uniform(256, 256) / 3.8 - 0.5 / 3.8
    det, det_thr = oracle.determinant(d), oracle.thr_determinant(d)
    assert det != 0 and abs(det - det_thr) <= max(min(abs(det), abs(det_thr)) * 1e-10, 1e-10)
    a48 = r.uniform(48, 48) - 0.5
    b = r.uniform(48, 3) - 0.5
    rc1, x1 = oracle.lineq_solve(a48, b)
    rc2, x2 = oracle.thr_lineq_solve(a48, b)
    assert rc1 == rc2 == 0 and np.abs(x1 - x2).max() <= 1e-4
    np.testing.assert_allclose(a48 @ x1, b, atol=1e-12)


def test_refinement_quirk_flag():
    # MatrixLinEQSolve's residual walks x along a row (LinAlgLU.pas:567): with k = 1 and an 8-byte
    # X stride both readings agree; with k > 1 only the column reading is a refinement.
    r = oracle.Mersenne(seed=3)
    a = r.uniform(40, 40) + 40 * np.eye(40)
    b = r.uniform(40, 1)
    _, xq = oracle.lineq_solve(a, b, 2, row_quirk=True)
    _, xc = oracle.lineq_solve(a, b, 2, row_quirk=False)
    assert np.array_equal(xq, xc)
    b3 = r.uniform(40, 3)
    _, xc3 = oracle.lineq_solve(a, b3, 2, row_quirk=False)
    assert oracle.backward_error(a, xc3, b3) < 1e-15


def test_backward_error_and_dot2():
    r = oracle.Mersenne(seed=11)
    a = r.uniform(200, 200)
    b = r.uniform(200, 2)
    _, x = oracle.lineq_solve(a, b)
    eta = oracle.backward_error(a, x, b)
    assert 0 <= eta < 200 * 2.0 ** -53
    # Dot2 residual of an exact integer system is exactly zero
    ai = np.round(r.uniform(30, 30) * 8)
    xi = np.round(r.uniform(30, 1) * 8)
    bi = ai @ xi
    assert np.all(oracle.residual_dot2(ai, xi, bi) == 0.0)


def test_singular_zero_column_and_nan():
    a = np.eye(5)
    a[:, 2] = 0.0
    rc, _ = oracle.lu_decomp_inplace(a.copy())
    assert rc == 1
    assert oracle.determinant(a) == 0.0


def _cx(pairs):
    return np.array([[complex(re, im) for re, im in row] for row in pairs])


def test_complex_lu_kats():
    """TestCmplx.pas: TestLU (:616-631, bitwise), TestLU2 (:633-662, MT seed 12705677, last element
    (486.05324, 9.5027968) within 1e-4), TestMtxInverse (:664-705, singular all-ones matrix, first
    row of the reference inverse within 1e-5) and TestDeterminant (:516-552, 33120 + 4608i)."""
    a = _cx([[(1.0, -1.0), (0.0, -1.0)], [(0.0, 2.0), (2.0, -1.0)]])
    rc, idx = oracle.cplx_lu_decomp_inplace(a)
    assert rc == 0 and a.tobytes() == _cx([[(1.0, -1.0), (0.0, -1.0)], [(-1.0, 1.0), (1.0, -2.0)]]).tobytes()
    r = oracle.Mersenne(seed=12705677)
    vals = [complex((r.u32() & 0x7FFFFFFF) % 200, (r.u32() & 0x7FFFFFFF) % 100) for _ in range(127 * 127)]
    x = np.array(vals).reshape(127, 127)
    rc, _ = oracle.cplx_lu_decomp_inplace(x)
    assert rc == 0 and abs(x[-1, -1] - (486.05324 + 9.5027968j)) <= 1e-4
    assert oracle.cplx_inverse_inplace(np.full((4, 4), 1 + 1j)) == 1
    v = np.array([complex(i, i + 1) for i in range(16)])
    v[::3] = -v[::3]
    a4 = v.reshape(4, 4)
    inv = a4.copy()
    assert oracle.cplx_inverse_inplace(inv) == 0
    np.testing.assert_allclose(inv[0], [0.242950984513183 - 0.232956465478163j, 0.027322404371585 - 0.032786885245902j,
                                        0.007541478129713 - 0.008295625942685j, -0.041420435345218 + 0.025207287622910j],
                               atol=1e-5)
    det = oracle.cplx_determinant(a4)
    assert abs(det - (33120 + 4608j)) <= 1e-12 * abs(det)


CHOL_A = np.array([[1.0, 2, 2], [-1, 4, -2], [2, 2, -1]])
CHOL_A2 = np.array([[1.0, 2, 2, 0.5], [-1, 4, -2, -0.1], [2, 2, -1, 1.2], [3, 2, -1, -1.1]])


def test_cholesky_kats():
    """TestCholesky (TestLineEquations.pas:494-524): X = A A^T factors (NR form), A itself does not,
    and the solve of X x = (2, -1, -1) gives (0.338888889, 0.00555555556, -0.2666666667)."""
    x = oracle.matrix_mult(CHOL_A, np.ascontiguousarray(CHOL_A.T))
    p = np.zeros((3, 4))  # LineWidthP = 4 doubles
    assert oracle.cholesky_nr(x, p) == 0
    assert oracle.cholesky_nr(CHOL_A.copy(), np.zeros((3, 4))) == 1
    res = oracle.cholesky_solve_nr(x, p, np.array([[2.0], [-1.0], [-1.0]]))
    np.testing.assert_allclose(res.ravel(), [0.338888889, 0.00555555556, -0.2666666667], atol=1e-9)


def test_cholesky2_kats_and_forms_agree():
    """TestCholesky2 (:526-571): InPlace4 with 2-column panels and InPlace2 succeed on A A^T (3 x 3
    and 4 x 4) and agree; InPlace2 reports crNoPositiveDefinite on A itself."""
    for a in (CHOL_A, CHOL_A2):
        x = oracle.matrix_mult(a, np.ascontiguousarray(a.T))
        x4, x2 = x.copy(), x.copy()
        assert oracle.cholesky_inplace4(x4, 2) == 0 and oracle.cholesky_inplace2(x2) == 0
        np.testing.assert_allclose(np.tril(x4), np.tril(x2), rtol=1e-13, atol=1e-13)
        lo = np.tril(x2)
        np.testing.assert_allclose(lo @ lo.T, x, rtol=1e-13, atol=1e-12)
    assert oracle.cholesky_inplace2(CHOL_A.copy()) == 1


def test_cholesky3_differential():
    """TestCholesky3 (:573-631) at n = 400 instead of 2048: unblocked, panel-24 and panel-32 (the
    class default) forms of the same SPD matrix x x^T agree."""
    r = oracle.Mersenne(seed=15)
    x = r.uniform(400, 400)
    a = oracle.matrix_mult(x, np.ascontiguousarray(x.T))
    a2, a24, a32 = a.copy(), a.copy(), a.copy()
    assert oracle.cholesky_inplace2(a2) == 0
    assert oracle.cholesky_inplace4(a24, 24) == 0 and oracle.cholesky_inplace4(a32) == 0
    for b in (a24, a32):
        assert np.linalg.norm(np.tril(b) - np.tril(a2)) <= 1e-9 * np.linalg.norm(np.tril(a2))
    assert np.array_equal(np.triu(a32, 1), np.triu(a, 1))


def test_oracle_against_lapack_real_and_complex():
    """The oracle's solves, inverses and determinants against numpy's LAPACK (an independent
    implementation) on seeded Gaussian systems of odd orders: normwise agreement to rounding."""
    r = oracle.Mersenne(seed=4242)
    for n in (33, 97, 130):
        a = r.gaussian(n, n)
        b = r.gaussian(n, 3)
        rc, x = oracle.lineq_solve(a, b)
        assert rc == 0
        np.testing.assert_allclose(x, np.linalg.solve(a, b), rtol=0, atol=1e-11 * np.abs(x).max())
        inv = a.copy()
        assert oracle.inverse_inplace(inv) == 0
        ref = np.linalg.inv(a)
        assert np.linalg.norm(inv - ref) <= 1e-11 * np.linalg.norm(ref)
        sgn, logdet = np.linalg.slogdet(a)
        det = oracle.determinant(a)
        assert np.sign(det) == sgn and abs(np.log(abs(det)) - logdet) <= 1e-11 * max(1.0, abs(logdet))
        z = a + 1j * r.gaussian(n, n)
        zb = b + 1j * r.gaussian(n, 3)
        rc, zx = oracle.cplx_lineq_solve(z, zb)
        assert rc == 0
        zref = np.linalg.solve(z, zb)
        assert np.linalg.norm(zx - zref) <= 1e-11 * np.linalg.norm(zref)
        zdet = oracle.cplx_determinant(z)
        zref_det = np.linalg.det(z)
        assert abs(zdet - zref_det) <= 1e-10 * abs(zref_det)


def test_oracle_cholesky_against_lapack():
    """The oracle's blocked Cholesky (MatrixCholeskyInPlace4) against numpy's LAPACK potrf on a
    seeded SPD matrix x x^T + n I."""
    r = oracle.Mersenne(seed=99)
    n = 150
    x = r.gaussian(n, n)
    a = x @ x.T + n * np.eye(n)
    f = a.copy()
    assert oracle.cholesky_inplace4(f, 32) == 0
    ref = np.linalg.cholesky(a)
    assert np.linalg.norm(np.tril(f) - ref) <= 1e-13 * np.linalg.norm(ref)
