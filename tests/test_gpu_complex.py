"""Complex LU (LinAlgLU.pas:1147-1603) through the C ABI against the oracle's restatement.

Bar: the reference's complex known answers (TestCmplx.pas: the 2 x 2 LU bitwise, the 127 x 127
MT-seeded LU's last element, the 4 x 4 inverse and determinant, the singular all-ones matrix);
pivots bit-exact against the oracle; factors, solutions and inverses within 1e-12 relative."""
import numpy as np
import pytest

import oracle
from mrmath_b200 import linalg as L

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def kat_4x4():
    """a[i] = (i, i+1), negated where i mod 3 = 0 (TestCmplx.pas:516-552, 664-705)."""
    v = np.array([complex(i, i + 1) for i in range(16)])
    v[::3] = -v[::3]
    return v.reshape(4, 4)


def cx(pairs):
    """complex128 array from (real, imag) pairs, so that zeros keep their sign as written"""
    return np.array([[complex(re, im) for re, im in row] for row in pairs])


def test_complex_lu_kat_2x2_bitwise(ctx):
    """TestLU (TestCmplx.pas:616-631): CheckEqualsMem against B."""
    a = cx([[(1.0, -1.0), (0.0, -1.0)], [(0.0, 2.0), (2.0, -1.0)]])
    st, idx = L.CplxMatrixLUDecompInPlace(a, ctx=ctx)
    assert st == 0
    assert a.tobytes() == cx([[(1.0, -1.0), (0.0, -1.0)], [(-1.0, 1.0), (1.0, -2.0)]]).tobytes()


def test_complex_lu_kat_127(ctx):
    """TestLU2 (TestCmplx.pas:633-662): MT19937 seed 12705677, re = RandInt(200), im = RandInt(100)."""
    r = oracle.Mersenne(seed=12705677)
    n = 127
    vals = np.empty(n * n, dtype=np.complex128)
    for i in range(n * n):
        re = (r.u32() & 0x7FFFFFFF) % 200
        im = (r.u32() & 0x7FFFFFFF) % 100
        vals[i] = complex(re, im)
    a = vals.reshape(n, n)
    ref = a.copy()
    rc0, i0 = oracle.cplx_lu_decomp_inplace(ref)
    st, idx = L.CplxMatrixLUDecompInPlace(a, ctx=ctx)
    assert st == rc0 == 0 and np.array_equal(idx, i0)
    for x in (a[-1, -1], ref[-1, -1]):
        assert abs(x.real - 486.05324) <= 1e-4 and abs(x.imag - 9.5027968) <= 1e-4, x
    assert rel(a, ref) <= RTOL


def test_complex_inverse_and_determinant_kats(ctx):
    ones = np.full((4, 4), 1 + 1j)
    o0 = ones.copy()
    assert L.CplxMatrixInverseInPlace(ones, ctx=ctx) == 1 and np.array_equal(ones, o0)
    a = kat_4x4()
    inv = a.copy()
    assert L.CplxMatrixInverseInPlace(inv, ctx=ctx) == 0
    ref = a.copy()
    assert oracle.cplx_inverse_inplace(ref) == 0
    assert rel(inv, ref) <= RTOL
    # cRefRes of TestMtxInverse (TestCmplx.pas:671-691), first row
    np.testing.assert_allclose(inv[0], [0.242950984513183 - 0.232956465478163j, 0.027322404371585 - 0.032786885245902j,
                                        0.007541478129713 - 0.008295625942685j, -0.041420435345218 + 0.025207287622910j],
                               atol=1e-5)
    det = L.CplxMatrixDeterminant(a, ctx=ctx)
    assert abs(det - (33120 + 4608j)) <= 1e-12 * abs(33120 + 4608j), det
    assert abs(det - oracle.cplx_determinant(a)) <= 1e-12 * abs(det)
    assert L.CplxMatrixDeterminant(o0, ctx=ctx) == 0


@pytest.mark.parametrize("n", [1, 2, 3, 31, 32, 33, 65, 100, 257, 600])
def test_complex_lu_solve_match_oracle(ctx, n):
    r = oracle.Mersenne(seed=900 + n)
    a = (r.uniform(n, n) - 0.5) + 1j * (r.uniform(n, n) - 0.5)
    b = (r.uniform(n, 3) - 0.5) + 1j * (r.uniform(n, 3) - 0.5)
    ref = a.copy()
    rc0, i0 = oracle.cplx_lu_decomp_inplace(ref)
    lu = a.copy()
    st, idx = L.CplxMatrixLUDecompInPlace(lu, ctx=ctx)
    assert st == rc0 == 0
    assert np.array_equal(idx, i0), np.nonzero(idx != i0)[0][:5]
    assert rel(lu, ref) <= RTOL
    st, x = L.CplxMatrixLinEQSolve(a, b, ctx=ctx)
    _, x_ref = oracle.cplx_lineq_solve(a, b)
    assert st == 0 and rel(x, x_ref) <= RTOL
    # back substitution with the reference-format factors and pivots
    y = b.copy()
    L.CplxMatrixLUBackSubst(lu, idx, y, ctx=ctx)
    assert rel(y, x_ref) <= RTOL


def test_complex_padded_strides_and_singular(ctx):
    n = 77
    r = oracle.Mersenne(seed=5)
    buf = (r.uniform(n, n + 3) - 0.5) + 1j * (r.uniform(n, n + 3) - 0.5)
    view = buf[:, :n]
    a = np.ascontiguousarray(view)
    pad = buf[:, n:].copy()
    st, idx = L.CplxMatrixLUDecompInPlace(view, ctx=ctx)
    ref = a.copy()
    _, i0 = oracle.cplx_lu_decomp_inplace(ref)
    assert st == 0 and np.array_equal(idx, i0) and rel(np.ascontiguousarray(view), ref) <= RTOL
    assert np.array_equal(buf[:, n:], pad)
    z = np.eye(6, dtype=np.complex128)
    z[:, 2] = 0
    st, _ = L.CplxMatrixLUDecompInPlace(z.copy(), ctx=ctx)
    assert st == 1 == oracle.cplx_lu_decomp_inplace(z.copy())[0]
