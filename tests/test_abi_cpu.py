"""CPU-side checks of the boundary: libb2m.so loads, exports exactly the entry points that
include/*.h declares, and the host mirror rejects bad arguments before any device work."""
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        names |= set(re.findall(r"B2M_API\s+[\w\s\*]+?\b(b2m_\w+)\s*\(", open(h).read()))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("b2m_create", "b2m_MatrixMultEx", "b2m_MatrixLUDecompInPlace", "b2m_MatrixLinEQSolve",
                 "b2m_MatrixLUBackSubst", "b2m_MatrixInverseInPlace", "b2m_MatrixDeterminant"):
        assert must in names


def test_library_exports_every_declared_symbol():
    import ctypes
    import mrmath_b200
    lib = ctypes.CDLL(mrmath_b200.LIB_PATH)
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_signatures_cover_header():
    from mrmath_b200 import _lib
    assert declared_symbols() <= set(_lib.SIGNATURES), set(declared_symbols()) - set(_lib.SIGNATURES)


def test_status_strings_without_gpu():
    from mrmath_b200 import _lib
    assert _lib.lib.b2m_status_string(1) == b"matrix is singular"
    assert _lib.lib.b2m_status_string(-1) == b"dimension error"
    # null context is rejected without touching a device
    assert _lib.lib.b2m_MatrixLUDecompInPlace(None, None, 0, 0, None) == _lib.ERR_ARG
