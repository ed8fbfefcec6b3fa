"""Error reports (b2m_MatrixMultErrorReport): the library's own compensated (Dot2) check of a
product, compared with the oracle's Dot2 rows of the same product."""
import numpy as np
import pytest

import oracle
from mrmath_b200 import inputs, linalg as L

pytestmark = pytest.mark.gpu


def _oracle_errors(c, a, b):
    ref, absab = oracle.gemm_rows_dot2(np.ascontiguousarray(a), np.ascontiguousarray(b), 0, a.shape[0])
    fwd = float(np.max(np.abs(c - ref)) / np.max(absab))
    relf = float(np.linalg.norm(c - ref) / np.linalg.norm(ref))
    return fwd, relf


@pytest.mark.parametrize("trans", [0, 1, 2])
def test_report_matches_oracle_dot2(ctx, trans):
    m, k, n = 130, 1000, 257
    a, b = inputs.c3_gauss_exp(m, k, n, seed=70 + trans)
    mt1 = a if trans != 1 else np.ascontiguousarray(a.T)
    mt2 = b if trans != 2 else np.ascontiguousarray(b.T)
    c = np.empty((m, n))
    L.MatrixMultEx(c, mt1, mt2, trans=trans, ctx=ctx)
    rep = L.MatrixMultErrorReport(c, mt1, mt2, trans=trans, sample_rows=m, ctx=ctx)
    assert rep["rows_checked"] == m and rep["bound"] == k * 2.0 ** -53
    fwd, relf = _oracle_errors(c, a, b)
    # both sides are compensated sums: they agree far below the errors they measure
    assert abs(rep["forward_error"] - fwd) <= 1e-3 * fwd + 1e-30, (rep, fwd)
    assert abs(rep["relative_error"] - relf) <= 1e-3 * relf + 1e-30, (rep, relf)
    assert rep["forward_error"] <= rep["bound"]


def test_report_sees_a_wrong_entry(ctx):
    a, b = inputs.c3_gauss_exp(64, 128, 96, seed=3)
    c = L.MatrixMult(a, b, ctx=ctx)
    clean = L.MatrixMultErrorReport(c, a, b, sample_rows=64, ctx=ctx)
    c[0, 5] += 1e-6 * np.max(np.abs(c))
    bad = L.MatrixMultErrorReport(c, a, b, sample_rows=64, ctx=ctx)
    assert bad["forward_error"] > 1e3 * clean["forward_error"]


def test_report_of_ozaki_and_dgemm_8192(ctx):
    """The GEMM benchmark's operands (m = n = k = 8192, g 2^e): both engines' products checked on
    the device against Dot2 rows."""
    import torch
    a, b = inputs.c3_gauss_exp(8192, 8192, 8192, seed=8)
    A, B = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    C = torch.empty((8192, 8192), dtype=torch.float64, device="cuda")
    L.dev_MatrixMultEx(C, A, B, ctx=ctx)
    rd = L.dev_MatrixMultErrorReport(C, A, B, sample_rows=32, ctx=ctx)
    L.dev_MatrixMultOzaki(C, A, B, slices=8, ctx=ctx)
    ro = L.dev_MatrixMultErrorReport(C, A, B, sample_rows=32, ctx=ctx)
    assert rd["rows_checked"] == 32 and rd["forward_error"] <= rd["bound"], rd
    assert rd["forward_error"] < 8e-15 and ro["forward_error"] < 8e-15, (rd, ro)
    assert ro["relative_error"] < 1e-12 and rd["relative_error"] < 1e-12, (rd, ro)
