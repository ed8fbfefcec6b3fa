"""mrmath_b200 -- B200 (sm_100a) implementation of mrMath's dense FP64 GEMM + pivoted-LU path.

The compute lives in libb2m.so (CUDA, C ABI in include/b2m.h).  This package only binds it:
`_lib` is the ctypes layer, `linalg` mirrors the reference's procedure-level API.
"""
from ._lib import B2MError, Context, LIB_PATH, lib  # noqa: F401  (raises if libb2m.so is missing)
from . import linalg  # noqa: F401
