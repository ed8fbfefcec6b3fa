"""mrmath_b200 -- B200 (sm_100a) implementation of mrMath's dense FP64 GEMM + pivoted-LU path.

The compute lives in libb2m.so (CUDA, C ABI in include/b2m.h).  This package only binds it:
`_lib` is the ctypes layer, `linalg` mirrors the reference's procedure-level API, `inputs` draws
the seeded synthetic workloads.  The shared library is loaded on first use of `_lib`, `linalg`,
`Context` or `lib` (importing `mrmath_b200.inputs` alone loads nothing), and loading raises if
libb2m.so is missing: there is no CPU fallback.
"""
import importlib

_FROM_LIB = ("B2MError", "Context", "LIB_PATH", "lib")


def __getattr__(name):
    if name in _FROM_LIB:
        return getattr(importlib.import_module("._lib", __name__), name)
    if name in ("linalg", "_lib", "autograd"):
        return importlib.import_module("." + name, __name__)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
