"""Seeded synthetic inputs for the five workloads, drawn from the reference's own generator.

numpy's legacy RandomState(seed) is MT19937 initialised with init_genrand(seed) -- the same state
as TRandomGenerator.InitMersenne (RandomEng.pas:626-644) -- and its random_sample() is the 53-bit
(a>>5 * 2^26 + b>>6) * 2^-53 of RandMersenneDbl (:749-765), its standard_normal() the Marsaglia
polar method of RandGauss (:283-307), returning and caching the two values in the same order.  The
test suite pins both streams element for element against the C restatement of the reference.

  c1_uniform   n = 1024 uniform [0,1) A and b (TDoubleMatrix.CreateRand, row-major fill)
  c2_kappa     A = U diag(s) V^T, s_i = kappa^(-i/(n-1)), U/V orthogonal factors of Gaussian
               matrices; 16 Gaussian right-hand sides
  c3_gauss_exp GEMM operands g * 2^e, g ~ N(0,1), e uniform integer in [-8, 8]
  c4_adjoint   A = R + n I, R uniform [-1,1); b, w Gaussian
  c5_batched   20,000 systems, n_i uniform integer [8, 256], A_i = R + n_i I, 1..4 Gaussian RHS
"""
from __future__ import annotations

import numpy as np


def rng(seed: int) -> np.random.RandomState:
    return np.random.RandomState(seed)


def c1_uniform(n: int = 1024, seed: int = 15):
    r = rng(seed)
    a = r.random_sample((n, n))
    b = r.random_sample((n, 1))
    return a, b


def _u32(r: np.random.RandomState, count: int) -> np.ndarray:
    # raw genrand_int32 outputs (RandMersenneDblWord): a full 32-bit range draws without rejection
    return r.randint(0, 2 ** 32, size=count, dtype=np.uint64).astype(np.uint32)


def c3_gauss_exp(m: int, k: int, n: int, seed: int = 15):
    """A (m x k) and B (k x n): all Gaussians of A, then all exponents of A, then the same for B;
    exponent = RandLW(17) - 8 = (genrand_int32 mod 17) - 8."""
    r = rng(seed)
    out = []
    for shape in ((m, k), (k, n)):
        g = r.standard_normal(shape)
        e = (_u32(r, g.size) % 17).astype(np.int64).reshape(shape) - 8
        out.append(np.ldexp(g, e))
    return out[0], out[1]


def c2_kappa(n: int = 8192, kappa: float = 1e5, nrhs: int = 16, seed: int = 15, device: str | None = None):
    """Returns (A, B) as torch float64 tensors on `device` (GPU QR for the orthogonal factors;
    the Q factors come from torch.linalg.qr of the seeded Gaussian matrices)."""
    import torch
    r = rng(seed)
    g1 = r.standard_normal((n, n))
    g2 = r.standard_normal((n, n))
    b = r.standard_normal((n, nrhs))
    dev = device or ("cuda" if torch.cuda.is_available() else "cpu")
    u, _ = torch.linalg.qr(torch.from_numpy(g1).to(dev))
    del g1
    v, _ = torch.linalg.qr(torch.from_numpy(g2).to(dev))
    del g2
    s = torch.tensor(kappa, dtype=torch.float64, device=dev) ** (
        -torch.arange(n, dtype=torch.float64, device=dev) / (n - 1))
    a = (u * s) @ v.T
    del u, v
    return a.contiguous(), torch.from_numpy(b).to(dev)


def c4_adjoint(n: int = 4096, seed: int = 15):
    r = rng(seed)
    a = 2.0 * r.random_sample((n, n)) - 1.0
    a[np.diag_indices(n)] += n
    b = r.standard_normal((n, 1))
    w = r.standard_normal((n, 1))
    return a, b, w


def c5_batched(count: int = 20000, lo: int = 8, hi: int = 256, seed: int = 15):
    """Lists of (A_i, B_i); sizes and RHS counts drawn first (uniform integers via
    genrand_int32 mod range), then each system's entries in order."""
    r = rng(seed)
    sizes = (_u32(r, count) % (hi - lo + 1)).astype(np.int64) + lo
    nrhs = (_u32(r, count) % 4).astype(np.int64) + 1
    mats, rhss = [], []
    for n, k in zip(sizes, nrhs):
        a = 2.0 * r.random_sample((n, n)) - 1.0
        a[np.diag_indices(n)] += n
        mats.append(a)
        rhss.append(r.standard_normal((n, k)))
    return sizes, nrhs, mats, rhss


def lu_solve_flops(n: int, nrhs: int) -> float:
    """LAPACK-convention flops of an LU solve: 2/3 n^3 + 2 n^2 nrhs."""
    return 2.0 / 3.0 * n ** 3 + 2.0 * n * n * nrhs
