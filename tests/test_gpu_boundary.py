"""Boundary features beyond the procedure calls: the progress callback (TLinEquProgress,
MatrixConst.pas:31, LinAlgLU.pas:272-276) and contexts on several devices."""
import numpy as np
import pytest

import oracle
from mrmath_b200 import linalg as L

pytestmark = pytest.mark.gpu


def test_progress_callback_reports_every_panel():
    import mrmath_b200
    c = mrmath_b200.Context(0)
    try:
        seen = []
        c.set_progress(seen.append)
        n = 300
        a = oracle.Mersenne(seed=300).uniform(n, n) - 0.5
        ref = a.copy()
        _, i0 = oracle.lu_decomp_inplace(ref)
        st, lu, idx = L.MatrixLUDecomp(a, ctx=c)
        assert st == 0 and np.array_equal(idx, i0)
        assert len(seen) >= (n + 31) // 32 and seen == sorted(seen) and seen[-1] == 100 and seen[0] > 0
        # a second call reports again from the start; removing the callback stops the reports
        seen.clear()
        st, x = L.MatrixLinEQSolve(a, np.ones((n, 1)), ctx=c)
        assert st == 0 and seen and seen[-1] == 100
        c.set_progress(None)
        seen.clear()
        L.MatrixLUDecomp(a, ctx=c)
        assert seen == []
    finally:
        c.close()


def test_resident_chain_and_sub_matrix_view(ctx):
    """Mult then SolveLinEQ on device-resident matrices (one upload per operand, one download),
    and a solve on a sub-matrix view of a larger resident matrix, against the oracle."""
    r = oracle.Mersenne(seed=77)
    n = 384
    # well-conditioned factors (kappa < 2 each) so that solutions can be held to 1e-12 against the
    # oracle: A = R1 - 0.5 + 2 sqrt(n) I and B = R2 - 0.5 + 2 sqrt(n) S, S the cyclic shift by 23
    # columns, so that the product's dominant entries C[i, i + 23] lie on the diagonal of the
    # 200 x 200 view at (17, 40) as well
    s = 2.0 * np.sqrt(n)
    a = r.uniform(n, n) - 0.5 + s * np.eye(n)
    b = r.uniform(n, n) - 0.5
    b[np.arange(n), (np.arange(n) + 23) % n] += s
    d = r.uniform(n, 3) - 0.5
    A, B, D = (L.ResidentMatrix.from_host(m, ctx=ctx) for m in (a, b, d))
    try:
        Cm = A.mult(B)
        st, X = Cm.solve(D)
        assert st == 0
        c_ref = np.zeros((n, n))
        oracle.block_mult(c_ref, a, b)
        assert np.abs(Cm.to_host() - c_ref).max() <= 4 * n * 2.0 ** -53 * np.abs(a).max() * np.abs(b).max() * n
        _, x_ref = oracle.lineq_solve(Cm.to_host(), d, row_quirk=False)
        x = X.to_host()
        assert np.linalg.norm(x - x_ref) <= 1e-12 * np.linalg.norm(x_ref)
        # a 200 x 200 block at (17, 40) of the resident product, solved in place of a copy
        V = Cm.sub(17, 40, 200, 200)
        rhs = L.ResidentMatrix.from_host(d[:200].copy(), ctx=ctx)
        st, Y = V.solve(rhs)
        assert st == 0
        blk = np.ascontiguousarray(Cm.to_host()[17:217, 40:240])
        _, y_ref = oracle.lineq_solve(blk, d[:200].copy(), row_quirk=False)
        assert np.linalg.norm(Y.to_host() - y_ref) <= 1e-12 * np.linalg.norm(y_ref)
        for m in (Cm, X, rhs, Y):
            m.free()
    finally:
        for m in (A, B, D):
            m.free()


def test_saved_matrix_straight_to_device(ctx, tmp_path):
    """A matrix saved in the reference's binary format is read into device memory and solved."""
    n = 257
    a = oracle.Mersenne(seed=257).uniform(n, n) - 0.5
    path = str(tmp_path / "a.bin")
    L.WriteMatrixFile(path, a)
    A, view = L.ResidentMatrix.from_file(path, ctx=ctx)
    assert view == {"sub_width": n, "sub_height": n, "offset_x": 0, "offset_y": 0}
    try:
        assert A.to_host().tobytes() == a.tobytes()
        b = L.ResidentMatrix.from_host(np.ones((n, 1)), ctx=ctx)
        st, X = A.solve(b)
        _, x_ref = oracle.lineq_solve(a, np.ones((n, 1)), row_quirk=False)
        assert st == 0 and np.linalg.norm(X.to_host() - x_ref) <= 1e-12 * np.linalg.norm(x_ref)
        b.free()
        X.free()
    finally:
        A.free()


def test_contexts_on_every_visible_device():
    """Launch attributes are set per device: a context on each visible device solves correctly."""
    import torch
    import mrmath_b200
    n = 700
    a = oracle.Mersenne(seed=701).uniform(n, n) - 0.5
    b = np.ones((n, 2))
    _, x_ref = oracle.lineq_solve(a, b, row_quirk=False)
    for dev in range(torch.cuda.device_count()):
        c = mrmath_b200.Context(dev)
        try:
            st, x = L.MatrixLinEQSolve(a, b, ctx=c)
            assert st == 0 and np.linalg.norm(x - x_ref) <= 1e-12 * np.linalg.norm(x_ref)
        finally:
            c.close()
