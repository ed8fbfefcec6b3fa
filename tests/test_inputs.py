"""The package's input generators draw the reference's own MT19937 streams (CPU only)."""
import numpy as np

import oracle
from mrmath_b200 import inputs


def test_uniform_and_gauss_streams_match_reference_generator():
    a = oracle.Mersenne(seed=15).uniform(50000)
    assert np.array_equal(a, inputs.rng(15).random_sample(50000))
    g = oracle.Mersenne(seed=15).gaussian(50001)
    assert np.array_equal(g, inputs.rng(15).standard_normal(50001))
    r = oracle.Mersenne(seed=15)
    u = np.array([r.u32() for _ in range(5000)], dtype=np.uint32)
    assert np.array_equal(u, inputs._u32(inputs.rng(15), 5000))


def test_c1_matches_createrand_fill():
    a, b = inputs.c1_uniform(64, seed=15)
    r = oracle.Mersenne(seed=15)
    assert np.array_equal(a, r.uniform(64, 64)) and np.array_equal(b, r.uniform(64, 1))


def test_c3_gauss_exp_matches_oracle():
    a, b = inputs.c3_gauss_exp(30, 20, 10, seed=4)
    r = oracle.Mersenne(seed=4)
    ra = r.gauss_exp(30, 20)
    rb = r.gauss_exp(20, 10)
    assert np.array_equal(a, ra) and np.array_equal(b, rb)
    e = np.frexp(a)[1]
    assert e.min() >= -12 and e.max() <= 14


def test_small_workload_shapes():
    s, k, mats, rhss = inputs.c5_batched(count=50, seed=3)
    assert len(mats) == 50 and s.min() >= 8 and s.max() <= 256 and k.min() >= 1 and k.max() <= 4
    assert all(m.shape == (n, n) and r.shape == (n, kk) for m, r, n, kk in zip(mats, rhss, s, k))
    a, b, w = inputs.c4_adjoint(64)
    assert np.all(np.diag(a) > 62)
    assert inputs.lu_solve_flops(8192, 16) == 2.0 / 3.0 * 8192 ** 3 + 2.0 * 8192 ** 2 * 16
