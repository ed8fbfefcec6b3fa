"""Ozaki split-precision GEMM (b2m_MatrixMultOzaki): FP64 products emulated with int8 slices on the
tcgen05 tensor cores, judged against the oracle's Dot2 (compensated) products.

Errors are reported normwise: max_ij |C - C_dot2| / max_ij (|A||B|)_ij, the quantity the native
DGEMM is also held to (its bound is ~K u)."""
import numpy as np
import pytest

import oracle
from mrmath_b200 import inputs, linalg as L

pytestmark = pytest.mark.gpu


def _fwd_err(c, a, b, rows=None):
    m = a.shape[0]
    if rows is None:
        ref, absab = oracle.gemm_rows_dot2(a, b, 0, m)
        got = c
    else:
        refs, abss, gots = [], [], []
        for r0 in rows:
            ref, absab = oracle.gemm_rows_dot2(a, b, int(r0), 1)
            refs.append(ref), abss.append(absab), gots.append(c[int(r0):int(r0) + 1])
        ref, absab, got = np.vstack(refs), np.vstack(abss), np.vstack(gots)
    return float(np.max(np.abs(got - ref)) / np.max(absab))


@pytest.mark.parametrize("m,k,n", [(200, 300, 130), (128, 128, 128), (257, 1000, 65), (1, 33, 7), (300, 4096, 300)])
def test_ozaki_matches_dot2(ctx, m, k, n):
    a, b = inputs.c3_gauss_exp(m, k, n, seed=m + k + n)
    c = L.MatrixMultOzaki(a, b, slices=8, ctx=ctx)
    err = _fwd_err(c, a, b)
    dg = L.MatrixMult(a, b, ctx=ctx)
    err_dgemm = _fwd_err(dg, a, b)
    # with a short K the native product is nearly exact and the slices' 2^-56 truncation of the
    # entries far below their row / column maximum (a 2^16 spread here) sets the floor
    assert err <= max(4 * err_dgemm, 2e-15), (err, err_dgemm)
    assert err < 8e-15


def test_ozaki_ops_and_slices(ctx):
    a, b = inputs.c3_gauss_exp(160, 520, 144, seed=3)
    ref, absab = oracle.gemm_rows_dot2(a, b, 0, a.shape[0])
    base = inputs.rng(9).standard_normal((160, 144))
    for op, sign in ((L.DO_ADD, 1.0), (L.DO_SUB, -1.0)):
        d = base.copy()
        L.MatrixMultOzaki(a, b, slices=8, dest=d, op=op, ctx=ctx)
        assert np.max(np.abs(d - (base + sign * ref))) / np.max(absab) < 8e-15
    # fewer slices: error grows by ~2^7 per slice dropped, and stays near the a-priori bound
    errs = {}
    for s in (3, 4, 6):
        errs[s] = float(np.max(np.abs(L.MatrixMultOzaki(a, b, slices=s, ctx=ctx) - ref)) / np.max(absab))
    assert errs[3] > errs[4] > errs[6]
    for s, e in errs.items():
        assert e < 2.0 ** (-7 * (s + 1) + 10 + 18), (s, e)  # 2^10 K-ish growth, 2^18 exponent spread


def test_ozaki_device_twin(ctx):
    import torch
    a, b = inputs.c3_gauss_exp(384, 512, 256, seed=5)
    A = torch.from_numpy(a).cuda()
    B = torch.from_numpy(b).cuda()
    C = torch.empty((384, 256), dtype=torch.float64, device="cuda")
    L.dev_MatrixMultOzaki(C, A, B, slices=8, ctx=ctx)
    torch.cuda.synchronize()
    assert _fwd_err(C.cpu().numpy(), a, b) < 8e-15


def test_ozaki_c3_8192(ctx):
    """The GEMM benchmark's shape and distribution, m = n = k = 8192, checked on 16 sampled rows."""
    import torch
    a, b = inputs.c3_gauss_exp(8192, 8192, 8192)
    A = torch.from_numpy(a).cuda()
    B = torch.from_numpy(b).cuda()
    C = torch.empty((8192, 8192), dtype=torch.float64, device="cuda")
    L.dev_MatrixMultOzaki(C, A, B, slices=8, ctx=ctx)
    torch.cuda.synchronize()
    rows = inputs.rng(1).randint(0, 8192, size=16)
    err = _fwd_err(C.cpu().numpy(), a, b, rows)
    L.dev_MatrixMultEx(C, A, B, ctx=ctx)
    torch.cuda.synchronize()
    err_dgemm = _fwd_err(C.cpu().numpy(), a, b, rows)
    assert err < 8e-15 and err <= max(4 * err_dgemm, 2e-15), (err, err_dgemm)
    # the native DGEMM (MatrixMult's drop-in) against the a-priori bound K u and the observed floor
    assert err_dgemm <= 8192 * 2.0 ** -53 and err_dgemm < 8e-15, err_dgemm
