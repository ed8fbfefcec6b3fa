"""ctypes binding of libb2m.so (the C ABI declared in include/b2m.h).

There is no fallback: if the shared library is missing or cannot be loaded, importing this
module raises, so nothing can silently run a CPU path in place of the CUDA one.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libb2m.so")

i32, i64, dbl, vp = C.c_int32, C.c_int64, C.c_double, C.c_void_p

# status codes (b2m.h)
OK, SINGULAR = 0, 1
ERR_DIM, ERR_CUDA, ERR_ALLOC, ERR_TIMEOUT, ERR_ARG, ERR_NOCONV, ERR_UNSUPPORTED = -1, -2, -3, -4, -5, -6, -7
ERR_FORMAT = -8
DO_NONE, DO_ADD, DO_SUB = 0, 1, 2
MIXED_TF32, MIXED_3XTF32 = 1, 3


class SolveReport(C.Structure):
    """b2m_solve_report"""
    _fields_ = [("iterations", C.c_int32), ("fell_back", C.c_int32), ("backward_error", C.c_double),
                ("refinement_backward_error", C.c_double), ("forward_error", C.c_double)]

class MatrixInfo(C.Structure):
    """b2m_matrix_info"""
    _fields_ = [("width", C.c_int64), ("height", C.c_int64), ("sub_width", C.c_int64), ("sub_height", C.c_int64),
                ("offset_x", C.c_int64), ("offset_y", C.c_int64)]


class GemmReport(C.Structure):
    """b2m_gemm_report"""
    _fields_ = [("rows_checked", C.c_int32), ("reserved", C.c_int32), ("forward_error", C.c_double),
                ("relative_error", C.c_double), ("bound", C.c_double)]


# name -> (restype, argtypes); pointers are passed as integers (c_void_p) so that numpy
# arrays (host) and torch tensors (device) use the same signatures.
SIGNATURES: dict[str, tuple] = {
    "b2m_create": (i32, [i32, C.POINTER(vp)]),
    "b2m_destroy": (i32, [vp]),
    "b2m_set_stream": (i32, [vp, vp]),
    "b2m_use_own_stream": (i32, [vp]),
    "b2m_use_graphs": (i32, [vp, i32]),
    "b2m_synchronize": (i32, [vp]),
    "b2m_set_wait_limit": (i32, [vp, i64]),
    "b2m_set_progress": (i32, [vp, vp, vp]),
    "b2m_ReadMatrixFile": (i32, [C.c_char_p, vp, vp, i64]),
    "b2m_dev_ReadMatrixFile": (i32, [vp, C.c_char_p, vp, vp, i64]),
    "b2m_WriteMatrixFile": (i32, [C.c_char_p, vp, i64, i64, i64]),
    "b2m_alloc": (i32, [vp, i64, i64, C.POINTER(vp), C.POINTER(i64)]),
    "b2m_free": (i32, [vp, vp]),
    "b2m_upload": (i32, [vp, vp, i64, vp, i64, i64, i64]),
    "b2m_download": (i32, [vp, vp, i64, vp, i64, i64, i64]),
    "b2m_last_error": (C.c_char_p, [vp]),
    "b2m_status_string": (C.c_char_p, [i32]),
    "b2m_kernel_launches": (i64, [vp]),
    "b2m_ctx_info": (i32, [vp, i32, C.POINTER(i64)]),
    "b2m_profile": (i32, [vp, i32]),
    "b2m_profile_read": (i32, [vp, i32, C.POINTER(i64), C.POINTER(dbl), C.POINTER(dbl)]),
    "b2m_MatrixMultEx": (i32, [vp, vp, i64, vp, vp, i64, i64, i64, i64, i64, i64, i32, i32]),
    "b2m_dev_MatrixMultEx": (i32, [vp, vp, i64, vp, vp, i64, i64, i64, i64, i64, i64, i32, i32]),
    "b2m_CplxMatrixLUDecompInPlace": (i32, [vp, vp, i64, i64, vp]),
    "b2m_CplxMatrixLUBackSubst": (i32, [vp, vp, i64, i64, vp, vp, i64, i64]),
    "b2m_CplxMatrixLinEQSolve": (i32, [vp, vp, i64, i64, vp, i64, vp, i64, i64]),
    "b2m_CplxMatrixInverseInPlace": (i32, [vp, vp, i64, i64]),
    "b2m_CplxMatrixDeterminant": (i32, [vp, vp, i64, i64, vp]),
    "b2m_MatrixCholeskyInPlace4": (i32, [vp, vp, i64, i64, i64]),
    "b2m_dev_MatrixCholeskyInPlace4": (i32, [vp, vp, i64, i64, vp]),
    "b2m_MatrixCholeskyInPlace": (i32, [vp, vp, i64, i64, vp, i64]),
    "b2m_MatrixCholeskySolveLinEq": (i32, [vp, vp, i64, i64, vp, i64, vp, i64, vp, i64, i64]),
    "b2m_dev_MatrixCholeskySolveLinEq": (i32, [vp, vp, i64, i64, vp, i64, vp, i64, vp, i64, i64]),
    "b2m_MatrixMultErrorReport": (i32, [vp, vp, i64, vp, vp, i64, i64, i64, i64, i64, i64, i32, i32, vp]),
    "b2m_dev_MatrixMultErrorReport": (i32, [vp, vp, i64, vp, vp, i64, i64, i64, i64, i64, i64, i32, i32, vp]),
    "b2m_MatrixLUDecompInPlace": (i32, [vp, vp, i64, i64, vp]),
    "b2m_MatrixLUDecomp": (i32, [vp, vp, i64, vp, i64, i64, vp]),
    "b2m_MatrixLUBackSubst": (i32, [vp, vp, i64, i64, vp, vp, i64, i64]),
    "b2m_MatrixInverseInPlace": (i32, [vp, vp, i64, i64]),
    "b2m_MatrixDeterminant": (i32, [vp, vp, i64, i64, vp]),
    "b2m_MatrixLinEQSolve": (i32, [vp, vp, i64, i64, vp, i64, vp, i64, i64, i64]),
    "b2m_dev_MatrixLUDecompInPlace": (i32, [vp, vp, i64, i64, vp, vp]),
    "b2m_dev_MatrixLUBackSubst": (i32, [vp, vp, i64, i64, vp, vp, i64, i64]),
    "b2m_dev_MatrixLinEQSolve": (i32, [vp, vp, i64, i64, vp, i64, vp, i64, i64, i64, vp]),
    "b2m_dev_MatrixInverseInPlace": (i32, [vp, vp, i64, i64, vp]),
    "b2m_dev_MatrixDeterminant": (i32, [vp, vp, i64, i64, vp]),
    "b2m_dev_MatrixLinEQSolveNoAlloc": (i32, [vp, vp, i64, i64, vp, i64, vp, i64, i64, vp]),
    "b2m_MatrixLinEQSolveMixed": (i32, [vp, vp, i64, i64, vp, i64, vp, i64, i64, i32, i32, dbl, vp]),
    "b2m_dev_MatrixLinEQSolveMixed": (i32, [vp, vp, i64, i64, vp, i64, vp, i64, i64, i32, i32, dbl, vp]),
    "b2m_MatrixMultOzaki": (i32, [vp, vp, i64, vp, vp, i64, i64, i64, i64, i64, i64, i32, i32]),
    "b2m_dev_MatrixMultOzaki": (i32, [vp, vp, i64, vp, vp, i64, i64, i64, i64, i64, i64, i32, i32]),
    "b2m_BatchLinEQSolve": (i32, [vp, i64, vp, vp, vp, vp, vp, vp, vp, i32, vp, vp]),
    "b2m_dev_BatchLinEQSolve": (i32, [vp, i64, vp, vp, vp, vp, vp, vp, vp, i32, vp, vp]),
    "b2m_batch_tune_read": (i32, [vp, vp, vp, vp, vp, vp]),
    "b2m_batch_tune_save": (i32, [vp, C.c_char_p]),
    "b2m_batch_tune_load": (i32, [vp, C.c_char_p, vp]),
    "b2m_MatrixLinEQSolveAdjoint": (i32, [vp, vp, i64, i64, vp, vp, i64, vp, i64, i64, vp, i64, vp, i64, i32]),
    "b2m_dev_MatrixLinEQSolveAdjoint": (i32, [vp, vp, i64, i64, vp, vp, i64, vp, i64, i64, vp, i64, vp, i64, i32]),
}


def load(path: str = LIB_PATH) -> C.CDLL:
    if not os.path.exists(path):
        raise ImportError(
            f"libb2m.so not found at {path}: build it with `python mrmath_b200/build.py` "
            "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = load()


class B2MError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"b2m status {status}: {msg}")
        self.status = status


class Context:
    """One libb2m context (device, stream, workspaces).  Mirrors b2m_create/b2m_destroy."""

    def __init__(self, device: int = 0):
        h = vp()
        st = lib.b2m_create(device, C.byref(h))
        if st != OK:
            raise B2MError(st, lib.b2m_status_string(st).decode())
        self.h = h
        self.device = device

    def close(self) -> None:
        if self.h:
            lib.b2m_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_error(self) -> str:
        return lib.b2m_last_error(self.h).decode()

    def check(self, status: int, allow=(OK,)) -> int:
        if status in allow:
            return status
        raise B2MError(status, f"{lib.b2m_status_string(status).decode()}: {self.last_error()}")

    def set_stream(self, stream_handle: int | None) -> None:
        """Bind a cudaStream_t (0 / None = the legacy default stream)."""
        self.check(lib.b2m_set_stream(self.h, stream_handle or None))

    def use_graphs(self, enable: bool) -> None:
        self.check(lib.b2m_use_graphs(self.h, int(enable)))

    def use_own_stream(self) -> None:
        self.check(lib.b2m_use_own_stream(self.h))

    def synchronize(self) -> None:
        self.check(lib.b2m_synchronize(self.h))

    PROGRESS_FN = C.CFUNCTYPE(None, C.c_int32, C.c_void_p)

    def set_progress(self, fn) -> None:
        """fn(percent) after every factored panel of the FP64 LU (TLinEquProgress); None removes it.
        It runs on a CUDA host thread and must not call this library."""
        self._progress = self.PROGRESS_FN(lambda pct, _user: fn(pct)) if fn is not None else None
        self.check(lib.b2m_set_progress(self.h, C.cast(self._progress, vp) if fn is not None else None, None))

    def set_wait_limit(self, polls: int) -> None:
        """Poll limit of the refinement sweeps' bounded waits (< 0: the built-in limit)."""
        self.check(lib.b2m_set_wait_limit(self.h, polls))

    def kernel_launches(self) -> int:
        return lib.b2m_kernel_launches(self.h)

    INFO_KEYS = {"num_sms": 1, "sweep_ctas": 2, "chain_clusters": 3, "chain_probe": 4, "chain_clusters4": 5,
                 "batch_big_warps": 6}

    def info(self, key: str) -> int:
        """b2m_ctx_info: an execution fact of this context (see INFO_KEYS)."""
        v = C.c_int64(0)
        self.check(lib.b2m_ctx_info(self.h, self.INFO_KEYS[key], C.byref(v)))
        return v.value

    KERNEL_CLASSES = ("gemm_f64", "panel", "row_swap", "trsm", "gemm_tc", "solve", "other")

    def profile(self, enable: bool) -> None:
        self.check(lib.b2m_profile(self.h, int(enable)))

    def profile_read(self) -> dict:
        out = {}
        for i, name in enumerate(self.KERNEL_CLASSES):
            n, ms, w = i64(0), dbl(0.0), dbl(0.0)
            self.check(lib.b2m_profile_read(self.h, i, C.byref(n), C.byref(ms), C.byref(w)))
            out[name] = {"launches": n.value, "ms": ms.value, "work": w.value}
        return out

    def lib_call(self, name: str, *args) -> int:
        """Raw status of a context entry point (no check)."""
        return getattr(lib, name)(self.h, *args)

    def call(self, name: str, *args, allow=(OK,)) -> int:
        return self.check(getattr(lib, name)(self.h, *args), allow=allow)
