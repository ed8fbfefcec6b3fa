"""Batched uneven solves (b2m_BatchLinEQSolve): every system against the oracle's restatement of
the reference's MatrixLinEQSolve, in both forms, with the edge orders of the size buckets."""
import numpy as np
import pytest

import oracle
from mrmath_b200 import inputs, linalg as L

pytestmark = pytest.mark.gpu

EDGE = [1, 2, 3, 7, 8, 15, 16, 17, 31, 32, 33, 63, 64, 65, 96, 127, 128, 129, 160, 200, 255, 256]


def _systems(seed, count, general_every=3):
    r = inputs.rng(seed)
    sizes = list(EDGE) + list(r.randint(1, 257, size=count - len(EDGE)))
    mats, rhss = [], []
    for i, n in enumerate(sizes):
        if i % general_every == 0:  # general matrix: pivoting matters
            a = r.random_sample((n, n))
        else:  # the benchmark's construction R + n I
            a = 2.0 * r.random_sample((n, n)) - 1.0
            a[np.diag_indices(n)] += n
        mats.append(a)
        rhss.append(r.standard_normal((n, int(r.randint(1, 9)))))
    return mats, rhss


def test_batch_plain_matches_oracle(ctx):
    mats, rhss = _systems(11, 150)
    xs, info, iters = L.BatchLinEQSolve(mats, rhss, mode=0, ctx=ctx)
    assert np.all(info == 0)
    for a, b, x in zip(mats, rhss, xs):
        rc, xr = oracle.lineq_solve(a, b, row_quirk=False)
        assert rc == 0
        err = np.linalg.norm(x - xr) / np.linalg.norm(xr)  # relative, normwise (Frobenius)
        assert err <= 1e-12, (a.shape[0], err)
        assert oracle.backward_error(a, x, b) <= 4 * a.shape[0] * 2.0 ** -53


def test_batch_mixed_reaches_fp64_backward_error(ctx):
    mats, rhss = _systems(12, 150)
    xs, info, iters = L.BatchLinEQSolve(mats, rhss, mode=1, ctx=ctx)
    assert np.all(info == 0)
    for a, b, x, it in zip(mats, rhss, xs, iters):
        eta = oracle.backward_error(a, x, b)
        assert eta <= a.shape[0] * 2.0 ** -53 or it == -1, (a.shape[0], eta, it)
    assert np.mean(iters >= 1) > 0.9  # almost every system converges without the FP64 fallback


def test_batch_singular_and_tiny(ctx):
    a1 = np.eye(5)
    a1[:, 2] = 0.0  # singular
    a2 = np.array([[2.0]])
    a3 = np.array([[0.0, 1.0], [1.0, 0.0]])  # needs the interchange
    mats = [a1, a2, a3]
    rhss = [np.ones((5, 1)), np.array([[4.0]]), np.array([[1.0, 2.0], [3.0, 4.0]])]
    for mode in (0, 1):
        xs, info, iters = L.BatchLinEQSolve(mats, rhss, mode=mode, ctx=ctx)
        assert list(info) == [1, 0, 0]
        assert np.allclose(xs[1], [[2.0]]) and np.allclose(xs[2], [[3.0, 4.0], [1.0, 2.0]])


def test_batch_device_twin_replay(ctx):
    import torch
    mats, rhss = _systems(13, 60)
    n, k, a_off, b_off, A, B = L.pack_batch(mats, rhss)
    dA = torch.from_numpy(A).cuda()
    dB = torch.from_numpy(B).cuda()
    outs = []
    for _ in range(2):
        dX = torch.zeros_like(dB)
        info = torch.full((len(n),), 7, dtype=torch.int32, device="cuda")
        L.dev_BatchLinEQSolve(n, k, a_off, b_off, dA, dB, dX, info, mode=0, ctx=ctx)
        torch.cuda.synchronize()
        assert int(info.max().item()) == 0
        outs.append(dX.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    xs = L.unpack_batch(outs[0], n, k, b_off)
    for a, b, x in zip(mats, rhss, xs):
        assert oracle.backward_error(a, x, b) <= 4 * a.shape[0] * 2.0 ** -53
    t = L.batch_tune(ctx)
    assert t["group_warps"] in (1, 2, 4) and t["pw_large"] in (8, 16, 32)


def test_autotune_table_persists_across_contexts(ctx, tmp_path):
    """The tuned tile shape of a plan, saved by one context and loaded by a fresh one, is reused
    (the second context launches the saved shape without timing the candidates) and gives the same
    answers."""
    import mrmath_b200
    mats, rhss = _systems(14, 40)
    xs, info, _ = L.BatchLinEQSolve(mats, rhss, mode=0, ctx=ctx)
    path = str(tmp_path / "tune.txt")
    L.batch_tune_save(path, ctx=ctx)
    shape = {k: v for k, v in L.batch_tune(ctx).items() if k != "ms"}
    c2 = mrmath_b200.Context(0)
    try:
        assert L.batch_tune_load(path, ctx=c2) >= 1
        launches0 = c2.kernel_launches()
        xs2, info2, _ = L.BatchLinEQSolve(mats, rhss, mode=0, ctx=c2)
        # no autotuning: one graph of one batch launch, not two launches per candidate shape
        assert c2.kernel_launches() - launches0 <= 2
        assert {k: v for k, v in L.batch_tune(c2).items() if k != "ms"} == shape
        assert np.array_equal(info, info2)
        for x, y in zip(xs, xs2):
            assert np.array_equal(x, y)
    finally:
        c2.close()
    bad = tmp_path / "bad.txt"
    bad.write_text("not a table\n")
    with pytest.raises(Exception):
        L.batch_tune_load(str(bad), ctx=ctx)
