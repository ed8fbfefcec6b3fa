"""ctypes front end of the CPU oracle (liboracle.so, built from mrmath_oracle.cpp).

TEST INFRASTRUCTURE ONLY.  The oracle restates mrMath's own FP64 GEMM / LU / solve / inverse /
determinant routines (src/LinAlgLU.pas, src/BlockedMult.pas, src/SimpleMatrixOperations.pas,
src/FMAMatrixMultTransposedOperationsx64.pas) and its MT19937 generator (src/RandomEng.pas).
Only tests/, the smoke check and bench.py's CPU-baseline leg use it, always as the checker or
the reported CPU baseline -- never as the product.

All matrices are numpy float64 arrays; strides are passed in bytes exactly as the reference's
LineWidth arguments, so padded views (a[:, :n] of a wider array) exercise the stride logic.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

_i32, _i64, _u32, _dbl = C.c_int32, C.c_int64, C.c_uint32, C.c_double
_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int32)


class Rng(C.Structure):
    _fields_ = [("mt", C.c_uint32 * 624), ("mti", C.c_int32), ("gauss_flag", C.c_int32), ("gauss2", C.c_double)]


def build() -> None:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load():
    if not os.path.exists(_LIB_PATH):
        build()
    lib = C.CDLL(_LIB_PATH)
    P = C.POINTER(Rng)
    sig = {
        "orc_rng_init": (None, [P, _i32]),
        "orc_rng_init_by_array": (None, [P, C.POINTER(_u32), _i32]),
        "orc_rng_u32": (_u32, [P]),
        "orc_rng_lw": (_u32, [P, _u32]),
        "orc_rng_dbl": (_dbl, [P]),
        "orc_rng_gauss": (_dbl, [P]),
        "orc_fill_uniform": (None, [P, _pd, _i64]),
        "orc_fill_gauss": (None, [P, _pd, _i64]),
        "orc_fill_gauss_exp": (None, [P, _pd, _i64]),
        "orc_set_mode": (None, [_i32]),
        "orc_get_mode": (_i32, []),
        "orc_matrix_mult": (None, [_pd, _i64, _pd, _pd] + [_i64] * 6),
        "orc_block_mult": (None, [_pd, _i64, _pd, _pd] + [_i64] * 7 + [_i32]),
        "orc_block_mult_t1": (None, [_pd, _i64, _pd, _pd] + [_i64] * 7 + [_i32]),
        "orc_block_mult_t2": (None, [_pd, _i64, _pd, _pd] + [_i64] * 7 + [_i32]),
        "orc_generic_mult": (None, [_pd, _i64, _pd, _pd] + [_i64] * 6),
        "orc_lu_decomp_inplace": (_i32, [_pd, _i64, _i64, _pi]),
        "orc_lu_decomp": (_i32, [_pd, _i64, _pd, _i64, _i64, _pi]),
        "orc_lu_backsubst": (None, [_pd, _i64, _i64, _pi, _pd, _i64]),
        "orc_inverse_inplace": (_i32, [_pd, _i64, _i64]),
        "orc_determinant": (_dbl, [_pd, _i64, _i64]),
        "orc_lineq_solve": (_i32, [_pd, _i64, _i64, _pd, _i64, _pd, _i64, _i64, _i64, _i32]),
        "orc_set_num_threads": (None, [_i32]),
        "orc_get_num_threads": (_i32, []),
        "orc_thr_matrix_mult": (None, [_pd, _i64, _pd, _pd] + [_i64] * 7 + [_i32]),
        "orc_thr_lu_decomp": (_i32, [_pd, _i64, _i64, _pi]),
        "orc_thr_lineq_solve": (_i32, [_pd, _i64, _i64, _pd, _i64, _pd, _i64, _i64, _i64]),
        "orc_thr_inverse": (_i32, [_pd, _i64, _i64]),
        "orc_thr_determinant": (_dbl, [_pd, _i64, _i64]),
        "orc_lu_min_pivot_gap": (_dbl, [_pd, _i64, _i64]),
        "orc_residual_dot2": (None, [_pd, _i64, _i64, _pd, _i64, _pd, _i64, _i64, _pd, _i64]),
        "orc_backward_error": (_dbl, [_pd, _i64, _i64, _pd, _i64, _pd, _i64, _i64]),
        "orc_gemm_rows_dot2": (None, [_pd, _i64, _pd, _i64, _i64, _i64, _i64, _i64, _i64, _pd, _i64, _pd, _i64]),
        "orc_cplx_lu_decomp_inplace": (_i32, [_pd, _i64, _i64, _pi]),
        "orc_cplx_lu_backsubst": (None, [_pd, _i64, _i64, _pi, _pd, _i64]),
        "orc_cplx_lineq_solve": (_i32, [_pd, _i64, _i64, _pd, _i64, _pd, _i64, _i64]),
        "orc_cplx_inverse_inplace": (_i32, [_pd, _i64, _i64]),
        "orc_cplx_determinant": (None, [_pd, _i64, _i64, _pd]),
        "orc_cholesky_inplace4": (_i32, [_pd, _i64, _i64, _i64]),
        "orc_cholesky_inplace2": (_i32, [_pd, _i64, _i64]),
        "orc_cholesky_nr": (_i32, [_pd, _i64, _i64, _pd, _i64]),
        "orc_cholesky_solve_nr": (None, [_pd, _i64, _i64, _pd, _i64, _pd, _i64, _pd, _i64]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def _p(a: np.ndarray):
    assert a.dtype == np.float64
    return a.ctypes.data_as(_pd)


def _pi32(a: np.ndarray):
    assert a.dtype == np.int32
    return a.ctypes.data_as(_pi)


def _lw(a: np.ndarray) -> int:
    """LineWidth in bytes of a 2-D row-major (possibly padded) view."""
    assert a.ndim == 2 and a.strides[1] == 8
    return a.strides[0]


# ------------------------------------------------------------------ random engine
class Mersenne:
    """TRandomGenerator with RandMethod = raMersenneTwister (src/RandomEng.pas)."""

    def __init__(self, seed: int | None = None, key: list[int] | None = None):
        self.state = Rng()
        self._p = C.byref(self.state)
        # fMTi = cN + 1 as after SetRandMethod (RandomEng.pas:401-402)
        self.state.mti = 625
        if key is not None:
            arr = (C.c_uint32 * len(key))(*key)
            lib.orc_rng_init_by_array(self._p, arr, len(key))
        elif seed is not None:
            lib.orc_rng_init(self._p, int(seed))

    def u32(self) -> int:
        return lib.orc_rng_u32(self._p)

    def lw(self, rng: int) -> int:
        return lib.orc_rng_lw(self._p, rng)

    def random(self) -> float:
        return lib.orc_rng_dbl(self._p)

    def gauss(self) -> float:
        return lib.orc_rng_gauss(self._p)

    def uniform(self, *shape) -> np.ndarray:
        out = np.empty(shape, dtype=np.float64)
        lib.orc_fill_uniform(self._p, _p(out), out.size)
        return out

    def gaussian(self, *shape) -> np.ndarray:
        out = np.empty(shape, dtype=np.float64)
        lib.orc_fill_gauss(self._p, _p(out), out.size)
        return out

    def gauss_exp(self, *shape) -> np.ndarray:
        out = np.empty(shape, dtype=np.float64)
        lib.orc_fill_gauss_exp(self._p, _p(out), out.size)
        return out


def set_mode(mode: str) -> None:
    lib.orc_set_mode(0 if mode == "generic" else 1)


def set_num_threads(n: int) -> None:
    lib.orc_set_num_threads(n)


def num_threads() -> int:
    return lib.orc_get_num_threads()


# ------------------------------------------------------------------ GEMM
def matrix_mult(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """MatrixMult (MatrixASMStubSwitch.pas:769-776)."""
    h1, w1 = a.shape
    h2, w2 = b.shape
    assert w1 == h2
    c = np.zeros((h1, w2))
    lib.orc_matrix_mult(_p(c), _lw(c), _p(a), _p(b), w1, h1, w2, h2, _lw(a), _lw(b))
    return c


def block_mult(c: np.ndarray, a: np.ndarray, b: np.ndarray, block: int = 128, op: int = 0, trans: int = 0) -> None:
    """In place: c (op)= op(a) * op(b).  trans 0 = A*B, 1 = A^T*B (T1), 2 = A*B^T (T2)."""
    h1, w1 = a.shape
    h2, w2 = b.shape
    f = {0: lib.orc_block_mult, 1: lib.orc_block_mult_t1, 2: lib.orc_block_mult_t2}[trans]
    f(_p(c), _lw(c), _p(a), _p(b), w1, h1, w2, h2, _lw(a), _lw(b), block, op)


def thr_block_mult(c: np.ndarray, a: np.ndarray, b: np.ndarray, block: int = 128, op: int = 0) -> None:
    h1, w1 = a.shape
    h2, w2 = b.shape
    lib.orc_thr_matrix_mult(_p(c), _lw(c), _p(a), _p(b), w1, h1, w2, h2, _lw(a), _lw(b), block, op)


# ------------------------------------------------------------------ LU path
def lu_decomp_inplace(a: np.ndarray, indx: np.ndarray | None = None) -> tuple[int, np.ndarray]:
    n = a.shape[1]
    if indx is None:
        indx = np.zeros(n, dtype=np.int32)
    rc = lib.orc_lu_decomp_inplace(_p(a), _lw(a), n, _pi32(indx))
    return rc, indx


def thr_lu_decomp_inplace(a: np.ndarray) -> tuple[int, np.ndarray]:
    n = a.shape[1]
    indx = np.zeros(n, dtype=np.int32)
    rc = lib.orc_thr_lu_decomp(_p(a), _lw(a), n, _pi32(indx))
    return rc, indx


def lu_backsubst(lu: np.ndarray, indx: np.ndarray, b: np.ndarray) -> None:
    """In place on b, which is an (n, k) view; only column 0 of the view is solved, like the reference."""
    n = lu.shape[1]
    lib.orc_lu_backsubst(_p(lu), _lw(lu), n, _pi32(indx), _p(b), _lw(b))


def inverse_inplace(a: np.ndarray) -> int:
    return lib.orc_inverse_inplace(_p(a), _lw(a), a.shape[1])


def thr_inverse_inplace(a: np.ndarray) -> int:
    return lib.orc_thr_inverse(_p(a), _lw(a), a.shape[1])


def determinant(a: np.ndarray) -> float:
    return lib.orc_determinant(_p(a), _lw(a), a.shape[1])


def thr_determinant(a: np.ndarray) -> float:
    return lib.orc_thr_determinant(_p(a), _lw(a), a.shape[1])


def lineq_solve(a: np.ndarray, b: np.ndarray, num_refinements: int = 0, row_quirk: bool = True):
    n = a.shape[1]
    k = b.shape[1]
    x = np.zeros((n, k))
    rc = lib.orc_lineq_solve(_p(a), _lw(a), n, _p(b), _lw(b), _p(x), _lw(x), k, num_refinements, int(row_quirk))
    return rc, x


def thr_lineq_solve(a: np.ndarray, b: np.ndarray, num_refinements: int = 0):
    n = a.shape[1]
    k = b.shape[1]
    x = np.zeros((n, k))
    rc = lib.orc_thr_lineq_solve(_p(a), _lw(a), n, _p(b), _lw(b), _p(x), _lw(x), k, num_refinements)
    return rc, x


def min_pivot_gap(a: np.ndarray) -> float:
    return lib.orc_lu_min_pivot_gap(_p(a), _lw(a), a.shape[1])


def residual_dot2(a: np.ndarray, x: np.ndarray, b: np.ndarray) -> np.ndarray:
    n = a.shape[1]
    k = b.shape[1]
    r = np.zeros((n, k))
    lib.orc_residual_dot2(_p(a), _lw(a), n, _p(x), _lw(x), _p(b), _lw(b), k, _p(r), _lw(r))
    return r


def backward_error(a: np.ndarray, x: np.ndarray, b: np.ndarray) -> float:
    """max_j ||b_j - A x_j||_inf / (||A||_inf ||x_j||_inf + ||b_j||_inf), residual in Dot2."""
    n = a.shape[1]
    return lib.orc_backward_error(_p(a), _lw(a), n, _p(x), _lw(x), _p(b), _lw(b), b.shape[1])


def gemm_rows_dot2(a: np.ndarray, b: np.ndarray, r0: int, nr: int):
    """Rows [r0, r0+nr) of A*B with Dot2 entries, plus the same rows of |A||B|."""
    m, k = a.shape
    _, n = b.shape
    c = np.zeros((nr, n))
    absab = np.zeros((nr, n))
    lib.orc_gemm_rows_dot2(_p(a), _lw(a), _p(b), _lw(b), m, n, k, r0, nr, _p(c), _lw(c), _p(absab), _lw(absab))
    return c, absab


# ------------------------------------------------------------------ Cholesky (LinAlgCholesky.pas)
def cholesky_inplace4(a: np.ndarray, pnl: int = 0) -> int:
    """MatrixCholeskyInPlace4 (TDoubleMatrix.Cholesky's routine): L in the lower triangle of a,
    the strict upper triangle left as it was.  0 = crOk, 1 = crNoPositiveDefinite."""
    return lib.orc_cholesky_inplace4(_p(a), _lw(a), a.shape[1], pnl)


def cholesky_inplace2(a: np.ndarray) -> int:
    return lib.orc_cholesky_inplace2(_p(a), _lw(a), a.shape[1])


def cholesky_nr(a: np.ndarray, p: np.ndarray) -> int:
    """MatrixCholeskyInPlace: L below the diagonal of a, its diagonal in p (an (n, k) view whose
    first column is used, like the reference's LineWidthP)."""
    return lib.orc_cholesky_nr(_p(a), _lw(a), a.shape[1], _p(p), _lw(p))


def cholesky_solve_nr(a: np.ndarray, p: np.ndarray, b: np.ndarray) -> np.ndarray:
    """MatrixCholeskySolveLinEq for one right-hand side column b (n, 1)."""
    x = np.zeros_like(b)
    lib.orc_cholesky_solve_nr(_p(a), _lw(a), a.shape[1], _p(p), _lw(p), _p(b), _lw(b), _p(x), _lw(x))
    return x


# ------------------------------------------------------------------ complex LU (LinAlgLU.pas:1147-1603)
def _pc(a: np.ndarray):
    assert a.dtype == np.complex128 and a.ndim == 2 and a.strides[1] == 16
    return a.ctypes.data_as(_pd)


def cplx_lu_decomp_inplace(a: np.ndarray) -> tuple[int, np.ndarray]:
    """CplxMatrixLUDecompInPlace on a complex128 array (TComplex = (real, imag) doubles)."""
    indx = np.zeros(a.shape[1], dtype=np.int32)
    rc = lib.orc_cplx_lu_decomp_inplace(_pc(a), a.strides[0], a.shape[1], _pi32(indx))
    return rc, indx


def cplx_lu_backsubst(lu: np.ndarray, indx: np.ndarray, b: np.ndarray) -> None:
    """CplxMatrixLUBackSubst in place on column 0 of b."""
    lib.orc_cplx_lu_backsubst(_pc(lu), lu.strides[0], lu.shape[1], _pi32(indx), _pc(b), b.strides[0])


def cplx_lineq_solve(a: np.ndarray, b: np.ndarray) -> tuple[int, np.ndarray]:
    x = np.zeros(b.shape, dtype=np.complex128)
    rc = lib.orc_cplx_lineq_solve(_pc(a), a.strides[0], a.shape[1], _pc(b), b.strides[0], _pc(x), x.strides[0],
                                  b.shape[1])
    return rc, x


def cplx_inverse_inplace(a: np.ndarray) -> int:
    return lib.orc_cplx_inverse_inplace(_pc(a), a.strides[0], a.shape[1])


def cplx_determinant(a: np.ndarray) -> complex:
    out = np.zeros(2)
    lib.orc_cplx_determinant(_pc(a), a.strides[0], a.shape[1], _p(out))
    return complex(out[0], out[1])
