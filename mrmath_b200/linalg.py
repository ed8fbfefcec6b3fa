"""Host-side mirror of the reference's procedure-level API for this path, over the C ABI.

Names and argument meaning follow the reference: MatrixMult / MatrixMultEx / MatrixMultT1Ex /
MatrixMultT2Ex (MatrixASMStubSwitch.pas:769-863), MatrixLUDecompInPlace, MatrixLUDecomp,
MatrixLUBackSubst, MatrixInverseInPlace, MatrixDeterminant, MatrixLinEQSolve (LinAlgLU.pas:26-45).
Matrices are numpy float64 2-D arrays (row-major; padded views such as a[:, :n] of a wider
array pass their row stride as the LineWidth).  Results use the reference's codes:
0 = leOk, 1 = leSingular.

`dev_*` functions take torch CUDA tensors and run asynchronously on torch's current stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import (DO_ADD, DO_NONE, DO_SUB, MIXED_3XTF32, MIXED_TF32, OK, SINGULAR, B2MError, Context, GemmReport,
                   SolveReport)

__all__ = [
    "default_context", "MatrixMult", "MatrixMultEx", "MatrixMultT1Ex", "MatrixMultT2Ex", "MatrixLUDecompInPlace",
    "MatrixLUDecomp", "MatrixLUBackSubst", "MatrixInverseInPlace", "MatrixDeterminant", "MatrixLinEQSolve",
    "MatrixLinEQSolveMixed", "MatrixLinEQSolveAdjoint", "DO_NONE", "DO_ADD", "DO_SUB",
]

_ctx: dict[int, Context] = {}


def default_context(device: int = 0) -> Context:
    c = _ctx.get(device)
    if c is None:
        c = _ctx[device] = Context(device)
    return c


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _lw(a: np.ndarray) -> int:
    if a.ndim != 2 or a.dtype != np.float64 or a.strides[1] != 8:
        raise ValueError("expected a 2-D float64 row-major array (rows may be padded)")
    return a.strides[0]


def _ctx_of(ctx):
    return ctx if ctx is not None else default_context()


# ----------------------------------------------------------------------------- GEMM
def MatrixMultEx(dest: np.ndarray, mt1: np.ndarray, mt2: np.ndarray, op: int = DO_NONE, trans: int = 0,
                 ctx: Context | None = None) -> None:
    """dest op= op(mt1) * op(mt2); trans 0: A*B, 1: A^T*B (T1), 2: A*B^T (T2)."""
    c = _ctx_of(ctx)
    h1, w1 = mt1.shape
    h2, w2 = mt2.shape
    c.call("b2m_MatrixMultEx", _ptr(dest), _lw(dest), _ptr(mt1), _ptr(mt2), w1, h1, w2, h2, _lw(mt1), _lw(mt2),
           op, trans)


def MatrixMultOzaki(mt1: np.ndarray, mt2: np.ndarray, slices: int = 8, dest: np.ndarray | None = None,
                    op: int = DO_NONE, ctx: Context | None = None) -> np.ndarray:
    """mt1 * mt2 in FP64 emulated on the INT8 tensor cores with `slices` 7-bit slices per operand."""
    h1, w1 = mt1.shape
    h2, w2 = mt2.shape
    if dest is None:
        dest = np.zeros((h1, w2))
    _ctx_of(ctx).call("b2m_MatrixMultOzaki", _ptr(dest), _lw(dest), _ptr(mt1), _ptr(mt2), w1, h1, w2, h2, _lw(mt1),
                      _lw(mt2), op, slices)
    return dest


def MatrixMult(mt1: np.ndarray, mt2: np.ndarray, ctx: Context | None = None) -> np.ndarray:
    dest = np.empty((mt1.shape[0], mt2.shape[1]))
    MatrixMultEx(dest, mt1, mt2, DO_NONE, 0, ctx)
    return dest


def _grep(rep) -> dict:
    return {"rows_checked": rep.rows_checked, "forward_error": rep.forward_error,
            "relative_error": rep.relative_error, "bound": rep.bound}


def MatrixMultErrorReport(dest: np.ndarray, mt1: np.ndarray, mt2: np.ndarray, trans: int = 0, sample_rows: int = 16,
                          ctx: Context | None = None) -> dict:
    """Error of a product dest = op(mt1) op(mt2) on sampled rows against the Dot2 product."""
    h1, w1 = mt1.shape
    h2, w2 = mt2.shape
    rep = GemmReport()
    _ctx_of(ctx).call("b2m_MatrixMultErrorReport", _ptr(dest), _lw(dest), _ptr(mt1), _ptr(mt2), w1, h1, w2, h2,
                      _lw(mt1), _lw(mt2), trans, sample_rows, C.addressof(rep))
    return _grep(rep)


def MatrixMultT1Ex(dest, mt1, mt2, op=DO_NONE, ctx=None):
    MatrixMultEx(dest, mt1, mt2, op, 1, ctx)


def MatrixMultT2Ex(dest, mt1, mt2, op=DO_NONE, ctx=None):
    MatrixMultEx(dest, mt1, mt2, op, 2, ctx)


# ----------------------------------------------------------------------------- LU
def MatrixLUDecompInPlace(A: np.ndarray, indx: np.ndarray | None = None, ctx: Context | None = None):
    n = A.shape[1]
    if indx is None:
        indx = np.zeros(n, dtype=np.int32)
    st = _ctx_of(ctx).call("b2m_MatrixLUDecompInPlace", _ptr(A), _lw(A), n, indx.ctypes.data, allow=(OK, SINGULAR))
    return st, indx


def MatrixLUDecomp(A: np.ndarray, ctx: Context | None = None):
    n = A.shape[1]
    LU = np.empty((n, n))
    indx = np.zeros(n, dtype=np.int32)
    st = _ctx_of(ctx).call("b2m_MatrixLUDecomp", _ptr(A), _lw(A), _ptr(LU), _lw(LU), n, indx.ctypes.data,
                           allow=(OK, SINGULAR))
    return st, LU, indx


def MatrixLUBackSubst(LU: np.ndarray, indx: np.ndarray, B: np.ndarray, ctx: Context | None = None) -> None:
    """Solves in place on every column of B (the reference solves one column per call)."""
    n = LU.shape[1]
    assert indx.dtype == np.int32
    _ctx_of(ctx).call("b2m_MatrixLUBackSubst", _ptr(LU), _lw(LU), n, indx.ctypes.data, _ptr(B), _lw(B), B.shape[1])


def MatrixInverseInPlace(A: np.ndarray, ctx: Context | None = None) -> int:
    return _ctx_of(ctx).call("b2m_MatrixInverseInPlace", _ptr(A), _lw(A), A.shape[1], allow=(OK, SINGULAR))


def MatrixDeterminant(A: np.ndarray, ctx: Context | None = None) -> float:
    det = C.c_double(0.0)
    _ctx_of(ctx).call("b2m_MatrixDeterminant", _ptr(A), _lw(A), A.shape[1], C.addressof(det))
    return det.value


def MatrixLinEQSolve(A: np.ndarray, B: np.ndarray, num_refinements: int = 0, X: np.ndarray | None = None,
                     ctx: Context | None = None):
    n = A.shape[1]
    k = B.shape[1]
    if X is None:
        X = np.zeros((n, k))
    st = _ctx_of(ctx).call("b2m_MatrixLinEQSolve", _ptr(A), _lw(A), n, _ptr(B), _lw(B), _ptr(X), _lw(X), k,
                           num_refinements, allow=(OK, SINGULAR))
    return st, X


def _rep(rep) -> dict:
    return {"iterations": rep.iterations, "fell_back": rep.fell_back, "backward_error": rep.backward_error,
            "refinement_backward_error": rep.refinement_backward_error, "forward_error": rep.forward_error}


def MatrixLinEQSolveMixed(A: np.ndarray, B: np.ndarray, mode: int = MIXED_3XTF32, max_iter: int = 0,
                          tol: float = 0.0, X: np.ndarray | None = None, ctx: Context | None = None):
    """FP32 tensor-core factorisation + FP64 refinement; returns (status, X, report)."""
    n = A.shape[1]
    k = B.shape[1]
    if X is None:
        X = np.zeros((n, k))
    rep = SolveReport()
    st = _ctx_of(ctx).call("b2m_MatrixLinEQSolveMixed", _ptr(A), _lw(A), n, _ptr(B), _lw(B), _ptr(X), _lw(X), k,
                           mode, max_iter, tol, C.addressof(rep), allow=(OK, SINGULAR))
    return st, X, _rep(rep)


def MatrixLinEQSolveAdjoint(LU: np.ndarray, indx: np.ndarray, X: np.ndarray, G: np.ndarray,
                            dA: np.ndarray | None = None, op: int = DO_NONE, ctx: Context | None = None):
    """Adjoint of MatrixLinEQSolve from the factors of MatrixLUDecomp: returns Lambda = A^-T G and
    fills dA with -Lambda X^T (op DO_NONE) or subtracts Lambda X^T from it (op DO_ADD)."""
    n = LU.shape[1]
    k = X.shape[1]
    assert indx.dtype == np.int32
    lam = np.empty((n, k))
    _ctx_of(ctx).call("b2m_MatrixLinEQSolveAdjoint", _ptr(LU), _lw(LU), n, indx.ctypes.data, _ptr(X), _lw(X),
                      _ptr(G), _lw(G), k, _ptr(lam), _lw(lam), _ptr(dA) if dA is not None else None,
                      _lw(dA) if dA is not None else 0, op)
    return lam


# ----------------------------------------------------------------------------- device (torch) twins
def _tptr(t) -> int:
    return t.data_ptr()


def _tlw(t) -> int:
    assert t.dim() == 2 and t.stride(1) == 1 and t.dtype.itemsize == 8
    return t.stride(0) * 8


def _bind_stream(c: Context, t) -> None:
    import torch
    c.set_stream(torch.cuda.current_stream(t.device).cuda_stream)


def dev_MatrixMultEx(dest, mt1, mt2, op=DO_NONE, trans=0, ctx=None):
    c = _ctx_of(ctx)
    _bind_stream(c, dest)
    h1, w1 = mt1.shape
    h2, w2 = mt2.shape
    c.call("b2m_dev_MatrixMultEx", _tptr(dest), _tlw(dest), _tptr(mt1), _tptr(mt2), w1, h1, w2, h2, _tlw(mt1),
           _tlw(mt2), op, trans)


def dev_MatrixLUDecompInPlace(A, indx, status=None, ctx=None):
    c = _ctx_of(ctx)
    _bind_stream(c, A)
    c.call("b2m_dev_MatrixLUDecompInPlace", _tptr(A), _tlw(A), A.shape[1], _tptr(indx),
           _tptr(status) if status is not None else None)


def dev_MatrixLUBackSubst(LU, indx, B, ctx=None):
    c = _ctx_of(ctx)
    _bind_stream(c, B)
    c.call("b2m_dev_MatrixLUBackSubst", _tptr(LU), _tlw(LU), LU.shape[1], _tptr(indx), _tptr(B), _tlw(B), B.shape[1])


def dev_MatrixLinEQSolve(A, B, X, num_refinements=0, status=None, ctx=None):
    c = _ctx_of(ctx)
    _bind_stream(c, A)
    c.call("b2m_dev_MatrixLinEQSolve", _tptr(A), _tlw(A), A.shape[1], _tptr(B), _tlw(B), _tptr(X), _tlw(X),
           B.shape[1], num_refinements, _tptr(status) if status is not None else None)


def dev_MatrixInverseInPlace(A, status=None, ctx=None):
    c = _ctx_of(ctx)
    _bind_stream(c, A)
    c.call("b2m_dev_MatrixInverseInPlace", _tptr(A), _tlw(A), A.shape[1],
           _tptr(status) if status is not None else None)


def dev_MatrixDeterminant(A, det, ctx=None):
    c = _ctx_of(ctx)
    _bind_stream(c, A)
    c.call("b2m_dev_MatrixDeterminant", _tptr(A), _tlw(A), A.shape[1], _tptr(det))


def dev_MatrixLinEQSolveMixed(A, B, X, mode=MIXED_3XTF32, max_iter=0, tol=0.0, status=None, ctx=None):
    """Device twin of MatrixLinEQSolveMixed; returns (status, report)."""
    c = _ctx_of(ctx)
    _bind_stream(c, A)
    rep = SolveReport()
    st = c.call("b2m_dev_MatrixLinEQSolveMixed", _tptr(A), _tlw(A), A.shape[1], _tptr(B), _tlw(B), _tptr(X), _tlw(X),
                B.shape[1], mode, max_iter, tol, C.addressof(rep), allow=(OK, SINGULAR))
    if status is not None:
        status.fill_(st)
    return st, _rep(rep)


def dev_MatrixLinEQSolveAdjoint(LU, indx, X, G, Lam, dA=None, op=DO_NONE, ctx=None):
    """Device twin of MatrixLinEQSolveAdjoint (torch CUDA tensors, indx int32 as produced by
    dev_MatrixLUDecompInPlace); Lam receives A^-T G, dA (optional) -Lam X^T."""
    c = _ctx_of(ctx)
    _bind_stream(c, LU)
    c.call("b2m_dev_MatrixLinEQSolveAdjoint", _tptr(LU), _tlw(LU), LU.shape[1], _tptr(indx), _tptr(X), _tlw(X),
           _tptr(G), _tlw(G), X.shape[1], _tptr(Lam), _tlw(Lam), _tptr(dA) if dA is not None else None,
           _tlw(dA) if dA is not None else 0, op)


# ----------------------------------------------------------------------------- batched uneven solves
def pack_batch(mats, rhss):
    """Packs lists of square A_i and B_i (n_i x k_i) into the flat layout of b2m_BatchLinEQSolve:
    returns (n, nrhs, a_off, b_off, A, B) with int32 orders / RHS counts and int64 offsets."""
    n = np.array([m.shape[0] for m in mats], dtype=np.int32)
    k = np.array([b.shape[1] for b in rhss], dtype=np.int32)
    a_sz = n.astype(np.int64) ** 2
    b_sz = n.astype(np.int64) * k
    a_off = np.concatenate([[0], np.cumsum(a_sz)[:-1]]).astype(np.int64)
    b_off = np.concatenate([[0], np.cumsum(b_sz)[:-1]]).astype(np.int64)
    A = np.concatenate([np.ascontiguousarray(m, dtype=np.float64).ravel() for m in mats])
    B = np.concatenate([np.ascontiguousarray(b, dtype=np.float64).ravel() for b in rhss])
    return n, k, a_off, b_off, A, B


def unpack_batch(X: np.ndarray, n, k, b_off):
    return [X[o:o + ni * ki].reshape(ni, ki) for ni, ki, o in zip(n, k, b_off)]


def BatchLinEQSolve(mats, rhss, mode: int = 0, ctx: Context | None = None):
    """Solves every A_i X_i = B_i in one batched launch; returns (list of X_i, info, iters)."""
    n, k, a_off, b_off, A, B = pack_batch(mats, rhss)
    X = np.zeros_like(B)
    info = np.zeros(len(n), dtype=np.int32)
    iters = np.zeros(len(n), dtype=np.int32)
    _ctx_of(ctx).call("b2m_BatchLinEQSolve", len(n), n.ctypes.data, k.ctypes.data, a_off.ctypes.data,
                      b_off.ctypes.data, _ptr(A), _ptr(B), _ptr(X), mode, info.ctypes.data, iters.ctypes.data)
    return unpack_batch(X, n, k, b_off), info, iters


def dev_BatchLinEQSolve(n, k, a_off, b_off, A, B, X, info, iters=None, mode: int = 0, ctx=None):
    """Device twin: plan arrays (numpy int32 / int64) on the host, A/B/X (flat float64) and
    info/iters (int32) torch CUDA tensors; asynchronous on torch's current stream."""
    c = _ctx_of(ctx)
    _bind_stream(c, A)
    c.call("b2m_dev_BatchLinEQSolve", len(n), n.ctypes.data, k.ctypes.data, a_off.ctypes.data, b_off.ctypes.data,
           _tptr(A), _tptr(B), _tptr(X), mode, _tptr(info), _tptr(iters) if iters is not None else None)


def batch_tune(ctx=None) -> dict:
    """The tile shape the batched solve's autotuner chose for the last plan."""
    vals = [C.c_int32(0) for _ in range(4)]
    ms = C.c_float(0.0)
    c = _ctx_of(ctx)
    c.call("b2m_batch_tune_read", *[C.addressof(v) for v in vals], C.addressof(ms))
    return {"small_n": vals[0].value, "group_warps": vals[1].value, "pw_large": vals[2].value,
            "pw_small": vals[3].value, "big_warps": c.info("batch_big_warps"), "ms": ms.value}


def batch_tune_save(path: str, ctx=None) -> None:
    """Writes the autotuner's table (every tuned batch plan and its tile shape) to `path`."""
    _ctx_of(ctx).call("b2m_batch_tune_save", path.encode())


def batch_tune_load(path: str, ctx=None) -> int:
    """Merges a saved autotuner table into the context; returns the number of plans taken."""
    n = C.c_int32(0)
    _ctx_of(ctx).call("b2m_batch_tune_load", path.encode(), C.addressof(n))
    return n.value


def dev_MatrixMultOzaki(dest, mt1, mt2, slices=8, op=DO_NONE, ctx=None):
    c = _ctx_of(ctx)
    _bind_stream(c, dest)
    h1, w1 = mt1.shape
    h2, w2 = mt2.shape
    c.call("b2m_dev_MatrixMultOzaki", _tptr(dest), _tlw(dest), _tptr(mt1), _tptr(mt2), w1, h1, w2, h2, _tlw(mt1),
           _tlw(mt2), op, slices)


def dev_MatrixMultErrorReport(dest, mt1, mt2, trans=0, sample_rows=16, ctx=None) -> dict:
    """Device twin of MatrixMultErrorReport (torch CUDA tensors); synchronizes the bound stream."""
    c = _ctx_of(ctx)
    _bind_stream(c, dest)
    h1, w1 = mt1.shape
    h2, w2 = mt2.shape
    rep = GemmReport()
    c.call("b2m_dev_MatrixMultErrorReport", _tptr(dest), _tlw(dest), _tptr(mt1), _tptr(mt2), w1, h1, w2, h2,
           _tlw(mt1), _tlw(mt2), trans, sample_rows, C.addressof(rep))
    return _grep(rep)


# ----------------------------------------------------------------------------- saved matrices
def ReadMatrixFile(path: str) -> tuple[np.ndarray, dict]:
    """ReadObjFromFile of a saved TDoubleMatrix ("RMCLS" binary stream): (full matrix, view info)."""
    from ._lib import MatrixInfo, lib
    info = MatrixInfo()
    st = lib.b2m_ReadMatrixFile(path.encode(), C.addressof(info), None, 0)
    if st != OK:
        raise B2MError(st, f"{lib.b2m_status_string(st).decode()}: {path}")
    out = np.empty((info.height, info.width))
    st = lib.b2m_ReadMatrixFile(path.encode(), C.addressof(info), _ptr(out), max(out.strides[0], 8))
    if st != OK:
        raise B2MError(st, lib.b2m_status_string(st).decode())
    view = {"sub_width": info.sub_width, "sub_height": info.sub_height, "offset_x": info.offset_x,
            "offset_y": info.offset_y}
    return out, view


def WriteMatrixFile(path: str, a: np.ndarray) -> None:
    """SaveToFile(path, TBinaryReaderWriter) of a matrix (empty Name, the full matrix as its view)."""
    from ._lib import lib
    st = lib.b2m_WriteMatrixFile(path.encode(), _ptr(a), _lw(a), a.shape[1], a.shape[0])
    if st != OK:
        raise B2MError(st, f"{lib.b2m_status_string(st).decode()}: {path}")


# ----------------------------------------------------------------------------- complex LU
def _zlw(a: np.ndarray) -> int:
    if a.ndim != 2 or a.dtype != np.complex128 or a.strides[1] != 16:
        raise ValueError("expected a 2-D complex128 row-major array (rows may be padded)")
    return a.strides[0]


def CplxMatrixLUDecompInPlace(A: np.ndarray, ctx: Context | None = None):
    """CplxMatrixLUDecompInPlace (LinAlgLU.pas:1308-1320) on a complex128 array; (status, indx)."""
    indx = np.zeros(A.shape[1], dtype=np.int32)
    st = _ctx_of(ctx).call("b2m_CplxMatrixLUDecompInPlace", _ptr(A), _zlw(A), A.shape[1], indx.ctypes.data,
                           allow=(OK, SINGULAR))
    return st, indx


def CplxMatrixLUBackSubst(LU: np.ndarray, indx: np.ndarray, B: np.ndarray, ctx: Context | None = None) -> None:
    _ctx_of(ctx).call("b2m_CplxMatrixLUBackSubst", _ptr(LU), _zlw(LU), LU.shape[1], indx.ctypes.data, _ptr(B),
                      _zlw(B), B.shape[1])


def CplxMatrixLinEQSolve(A: np.ndarray, B: np.ndarray, ctx: Context | None = None):
    X = np.zeros(B.shape, dtype=np.complex128)
    st = _ctx_of(ctx).call("b2m_CplxMatrixLinEQSolve", _ptr(A), _zlw(A), A.shape[1], _ptr(B), _zlw(B), _ptr(X),
                           _zlw(X), B.shape[1], allow=(OK, SINGULAR))
    return st, X


def CplxMatrixInverseInPlace(A: np.ndarray, ctx: Context | None = None) -> int:
    return _ctx_of(ctx).call("b2m_CplxMatrixInverseInPlace", _ptr(A), _zlw(A), A.shape[1], allow=(OK, SINGULAR))


def CplxMatrixDeterminant(A: np.ndarray, ctx: Context | None = None) -> complex:
    det = np.zeros(2)
    _ctx_of(ctx).call("b2m_CplxMatrixDeterminant", _ptr(A), _zlw(A), A.shape[1], _ptr(det))
    return complex(det[0], det[1])


# ----------------------------------------------------------------------------- Cholesky
def MatrixCholeskyInPlace4(A: np.ndarray, pnl_size: int = 0, ctx: Context | None = None) -> int:
    """A = L L^T, L in A's lower triangle (LinAlgCholesky.pas:106-123); 0 = crOk, 1 = not positive definite."""
    return _ctx_of(ctx).call("b2m_MatrixCholeskyInPlace4", _ptr(A), _lw(A), A.shape[1], pnl_size, allow=(OK, 1))


def MatrixCholeskyInPlace(A: np.ndarray, P: np.ndarray, ctx: Context | None = None) -> int:
    """Numerical-Recipes form (LinAlgCholesky.pas:270-332): L below A's diagonal, the diagonal in P's
    first column (P an (n, k) array: element i at byte offset i * LineWidthP)."""
    return _ctx_of(ctx).call("b2m_MatrixCholeskyInPlace", _ptr(A), _lw(A), A.shape[1], _ptr(P), _lw(P),
                             allow=(OK, 1))


def MatrixCholeskySolveLinEq(A: np.ndarray, B: np.ndarray, P: np.ndarray | None = None,
                             ctx: Context | None = None) -> np.ndarray:
    """X with A X = B from a Cholesky factor (NR form with P, or the InPlace4 form without)."""
    n, k = A.shape[1], B.shape[1]
    X = np.zeros((n, k))
    _ctx_of(ctx).call("b2m_MatrixCholeskySolveLinEq", _ptr(A), _lw(A), n, _ptr(P) if P is not None else None,
                      _lw(P) if P is not None else 0, _ptr(B), _lw(B), _ptr(X), _lw(X), k)
    return X


def dev_MatrixCholeskyInPlace4(A, status=None, ctx=None):
    c = _ctx_of(ctx)
    _bind_stream(c, A)
    c.call("b2m_dev_MatrixCholeskyInPlace4", _tptr(A), _tlw(A), A.shape[1],
           _tptr(status) if status is not None else None)


def dev_MatrixCholeskySolveLinEq(A, B, X, P=None, ctx=None):
    c = _ctx_of(ctx)
    _bind_stream(c, A)
    c.call("b2m_dev_MatrixCholeskySolveLinEq", _tptr(A), _tlw(A), A.shape[1], _tptr(P) if P is not None else None,
           P.stride(0) * 8 if P is not None else 0, _tptr(B), _tlw(B), _tptr(X), _tlw(X), B.shape[1])


# ----------------------------------------------------------------------------- resident matrices
class ResidentMatrix:
    """A matrix kept in device memory across chained calls: the resident form a TDoubleMatrix
    subclass keeps (b2m_alloc / b2m_upload / b2m_download and the b2m_dev_* entry points on the
    context's own stream), without torch.  `sub` is a view into the parent (SetSubMatrix,
    Matrix.pas:70): same storage, the parent's LineWidth."""

    def __init__(self, ctx: Context, rows: int, cols: int, _view_of=None, _ptr=None, _lw=None):
        self.ctx, self.rows, self.cols = ctx, rows, cols
        self._parent = _view_of
        if _view_of is None:
            p, lw = C.c_void_p(), C.c_int64()
            ctx.check(ctx.lib_call("b2m_alloc", rows, cols, C.byref(p), C.byref(lw)))
            self.ptr, self.lw = p.value, lw.value
        else:
            self.ptr, self.lw = _ptr, _lw

    @classmethod
    def from_host(cls, a: np.ndarray, ctx: Context | None = None) -> "ResidentMatrix":
        c = _ctx_of(ctx)
        m = cls(c, a.shape[0], a.shape[1])
        c.check(c.lib_call("b2m_upload", m.ptr, m.lw, _ptr(a), _lw(a), a.shape[0], a.shape[1]))
        return m

    @classmethod
    def from_file(cls, path: str, ctx: Context | None = None) -> tuple["ResidentMatrix", dict]:
        """A saved TDoubleMatrix read straight into device memory (b2m_dev_ReadMatrixFile): the
        full matrix and its saved sub-matrix view (apply it with `sub`)."""
        from ._lib import MatrixInfo
        c = _ctx_of(ctx)
        info = MatrixInfo()
        c.check(c.lib_call("b2m_dev_ReadMatrixFile", path.encode(), C.addressof(info), None, 0))
        m = cls(c, info.height, info.width)
        c.check(c.lib_call("b2m_dev_ReadMatrixFile", path.encode(), C.addressof(info), m.ptr, m.lw))
        return m, {"sub_width": info.sub_width, "sub_height": info.sub_height, "offset_x": info.offset_x,
                   "offset_y": info.offset_y}

    def to_host(self) -> np.ndarray:
        out = np.empty((self.rows, self.cols))
        self.ctx.check(self.ctx.lib_call("b2m_download", _ptr(out), _lw(out), self.ptr, self.lw, self.rows,
                                         self.cols))
        return out

    def sub(self, r0: int, c0: int, rows: int, cols: int) -> "ResidentMatrix":
        if r0 < 0 or c0 < 0 or r0 + rows > self.rows or c0 + cols > self.cols:
            raise ValueError("sub-matrix outside the matrix")
        return ResidentMatrix(self.ctx, rows, cols, _view_of=self, _ptr=self.ptr + r0 * self.lw + c0 * 8,
                              _lw=self.lw)

    def mult(self, other: "ResidentMatrix", trans: int = 0) -> "ResidentMatrix":
        """op(self) * op(other) into a new resident matrix (MultEx with doNone)."""
        m = self.cols if trans == 1 else self.rows
        n = other.rows if trans == 2 else other.cols
        out = ResidentMatrix(self.ctx, m, n)
        self.ctx.use_own_stream()
        self.ctx.call("b2m_dev_MatrixMultEx", out.ptr, out.lw, self.ptr, other.ptr, self.cols, self.rows, other.cols,
                      other.rows, self.lw, other.lw, DO_NONE, trans)
        return out

    def solve(self, rhs: "ResidentMatrix") -> tuple[int, "ResidentMatrix"]:
        """SolveLinEQ: X with self X = rhs; returns (status, X)."""
        x = ResidentMatrix(self.ctx, rhs.rows, rhs.cols)
        st = ResidentMatrix(self.ctx, 1, 1)  # one int32 result word in the first bytes
        try:
            self.ctx.use_own_stream()
            self.ctx.call("b2m_dev_MatrixLinEQSolve", self.ptr, self.lw, self.cols, rhs.ptr, rhs.lw, x.ptr, x.lw,
                          rhs.cols, 0, st.ptr)
            word = st.to_host().view(np.int32)[0, 0]
        finally:
            st.free()
        return int(word), x

    def free(self) -> None:
        if self._parent is None and self.ptr:
            self.ctx.check(self.ctx.lib_call("b2m_free", self.ptr))
        self.ptr = 0
