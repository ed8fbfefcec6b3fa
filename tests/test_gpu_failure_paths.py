"""Every failure branch of the solves, driven on purpose and checked against the oracle.

* the mixed solve's FP64 fallback when refinement does not reach the tolerance (max_iter = 1 with
  an unreachable tolerance);
* the FP32 factorisation's tiny-pivot branch (entries below the FP32 normal range), which hands
  the system to the FP64 factorisation;
* a bounded wait that runs out: with a wait limit of 0 polls every dependent wait of the
  refinement sweeps gives up at once, the call returns B2M_ERR_TIMEOUT, and the same context then
  solves correctly with the built-in limit (no GPU fault, no hang: every wait is bounded);
* NaN and Inf entries: the plain LU must pick the pivots the reference's leaf picks
  (`Abs(x) > absMaxVal`, LinAlgLU.pas:246-256, never selects a NaN) and report the same status.
"""
import numpy as np
import pytest

import oracle
from mrmath_b200 import _lib, inputs, linalg as L

pytestmark = pytest.mark.gpu


def _dd_system(n, k, seed):
    r = inputs.rng(seed)
    a = r.random_sample((n, n)) - 0.5
    a[np.diag_indices(n)] += 2.0
    return a, r.standard_normal((n, k))


def test_forced_fp64_fallback(ctx):
    n, k = 700, 3
    a, b = _dd_system(n, k, 41)
    st, x, rep = L.MatrixLinEQSolveMixed(a, b, mode=_lib.MIXED_3XTF32, max_iter=1, tol=1e-300, ctx=ctx)
    assert st == 0 and rep["fell_back"] == 1 and rep["iterations"] == 1, rep
    eta = oracle.backward_error(a, x, b)
    assert eta <= n * 2.0 ** -53 and rep["backward_error"] <= n * 2.0 ** -53, (eta, rep)
    # the refinement's own last step is reported separately and was above the tolerance
    assert rep["refinement_backward_error"] > 1e-300
    _, x_ref = oracle.lineq_solve(a, b, row_quirk=False)
    assert np.linalg.norm(x - x_ref) <= 1e-12 * np.linalg.norm(x_ref)
    assert 0.0 <= rep["forward_error"] < 1e-10, rep


def test_fp32_tiny_pivot_falls_back_to_fp64(ctx):
    n, k = 300, 2
    a, b = _dd_system(n, k, 42)
    a *= 1e-40  # below FLT_MIN: the FP32 pivots are <= 10/FLT_MAX, FP64 handles it normally
    st, x, rep = L.MatrixLinEQSolveMixed(a, b, mode=_lib.MIXED_3XTF32, ctx=ctx)
    assert st == 0 and rep["fell_back"] == 1 and rep["iterations"] == 0, rep
    assert np.all(np.isfinite(x))
    assert oracle.backward_error(a, x, b) <= n * 2.0 ** -53
    _, x_ref = oracle.lineq_solve(a, b, row_quirk=False)
    assert np.linalg.norm(x - x_ref) <= 1e-12 * np.linalg.norm(x_ref)


def test_bounded_wait_runs_out_and_context_survives():
    import torch
    import mrmath_b200
    c = mrmath_b200.Context(0)
    try:
        n, k = 1024, 16
        a, b = _dd_system(n, k, 43)
        A, B = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
        X = torch.empty_like(B)
        c.set_wait_limit(0)
        with pytest.raises(_lib.B2MError) as ei:
            L.dev_MatrixLinEQSolveMixed(A, B, X, ctx=c)
        assert ei.value.status == _lib.ERR_TIMEOUT
        assert "bounded wait" in c.last_error()
        c.set_wait_limit(-1)
        st, rep = L.dev_MatrixLinEQSolveMixed(A, B, X, ctx=c)
        torch.cuda.synchronize()
        assert st == 0 and rep["fell_back"] == 0, rep
        assert oracle.backward_error(a, X.cpu().numpy(), b) <= n * 2.0 ** -53
    finally:
        c.close()


def _nan_case(n, where, value, seed):
    r = oracle.Mersenne(seed=seed)
    a = r.uniform(n, n) - 0.5
    for (i, j) in where:
        a[i, j] = value
    return a


@pytest.mark.parametrize("value", [np.nan, np.inf, -np.inf])
@pytest.mark.parametrize("n,where", [(64, [(40, 3)]), (96, [(0, 0)]), (300, [(200, 150), (17, 290)])])
def test_nan_inf_pivots_match_oracle(ctx, n, where, value):
    a = _nan_case(n, where, value, seed=n + len(where))
    ref = a.copy()
    rc0, i0 = oracle.lu_decomp_inplace(ref)
    st, lu, idx = L.MatrixLUDecomp(a, ctx=ctx)
    assert st == rc0
    if rc0 != 0:
        return
    assert np.array_equal(idx, i0), np.nonzero(idx != i0)[0][:5]
    assert np.array_equal(np.isnan(lu), np.isnan(ref))
    assert np.array_equal(np.isposinf(lu), np.isposinf(ref)) and np.array_equal(np.isneginf(lu), np.isneginf(ref))
    fin = np.isfinite(ref)
    assert np.linalg.norm(lu[fin] - ref[fin]) <= 1e-12 * np.linalg.norm(ref[fin])


def test_all_nan_column_is_singular(ctx):
    a = _nan_case(40, [(i, 5) for i in range(40)], np.nan, seed=7)
    rc0, _ = oracle.lu_decomp_inplace(a.copy())
    st, _ = L.MatrixLUDecompInPlace(a.copy(), ctx=ctx)
    assert rc0 == 1 and st == 1
