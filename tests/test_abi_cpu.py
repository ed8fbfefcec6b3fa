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


def test_reference_arm_loads_no_libb2m():
    """bench.py --impl reference times the oracle's restatement of the reference alone: the run
    (here on a small system) must not import the ctypes layer nor map libb2m.so."""
    import json
    import subprocess
    import sys
    code = (
        "import sys, json, argparse; sys.path.insert(0, %r); sys.argv = ['bench.py'];"
        "import bench;"
        "a = argparse.Namespace(n=96, nrhs=2, kappa=1e4, steps=2, warmup=1, gpus=1);"
        "bench.run_reference(a, 1, 0);"
        "maps = open('/proc/self/maps').read();"
        "print(json.dumps({'lib': 'mrmath_b200._lib' in sys.modules, 'mapped': 'libb2m.so' in maps}))" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True, timeout=600)
    lines = [json.loads(x) for x in out.stdout.strip().splitlines()]
    line, probe = lines[0], lines[-1]
    assert line["impl"] == "reference" and line["config"]["n"] == 96 and line["steps"] == 2
    assert line["backward_error"] <= 96 * 2.0 ** -53
    assert probe == {"lib": False, "mapped": False}


def test_status_strings_without_gpu():
    from mrmath_b200 import _lib
    assert _lib.lib.b2m_status_string(1) == b"matrix is singular"
    assert _lib.lib.b2m_status_string(-1) == b"dimension error"
    # null context is rejected without touching a device
    assert _lib.lib.b2m_MatrixLUDecompInPlace(None, None, 0, 0, None) == _lib.ERR_ARG


def _c_arg_count(args: str) -> int:
    args = re.sub(r"/\*.*?\*/", "", args, flags=re.S).strip()
    return 0 if args in ("", "void") else len(args.split(","))


def _pascal_arg_count(args: str) -> int:
    n = 0
    for group in args.split(";"):
        names = re.sub(r"^(out|var|const)\s+", "", group.split(":")[0].strip())
        n += len([x for x in names.split(",") if x.strip()])
    return n


def test_integration_bindings_match_header():
    """The Pascal unit and the ctypes stub in INTEGRATION.md bind only entry points that the header
    declares, each `cdecl; external` with the header's argument count."""
    header = "".join(open(h).read() for h in glob.glob(os.path.join(ROOT, "include", "*.h")))
    decl = {m.group(1): m.group(2) for m in
            re.finditer(r"B2M_API\s+[\w\s\*]+?\b(b2m_\w+)\s*\((.*?)\)\s*;", header, re.S)}
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    externals = re.findall(r"function\s+(b2m_\w+)\s*\((.*?)\)\s*:\s*\w+\s*;\s*cdecl;\s*external", doc, re.S)
    assert len(externals) >= 30
    for name, args in externals:
        assert name in decl, f"{name} bound in the Pascal unit but not declared"
        assert _pascal_arg_count(args) == _c_arg_count(decl[name]), name
    for name in set(re.findall(r"lib\.(b2m_\w+)", doc)):
        assert name in decl, f"{name} used by the ctypes stub but not declared"
    argtypes = re.search(r"lib\.b2m_MatrixLinEQSolve\.argtypes\s*=\s*\[(.*?)\]", doc, re.S).group(1)
    assert argtypes.count("ctypes.") == _c_arg_count(decl["b2m_MatrixLinEQSolve"])


def test_null_context_and_no_device_are_errors_not_crashes():
    """Every entry point that takes a context returns B2M_ERR_ARG for a null one (and null
    buffers) before it touches a device; b2m_create on a machine without a usable device returns
    B2M_ERR_CUDA and leaves the handle null.  Runs without a GPU."""
    import ctypes

    import torch

    from mrmath_b200 import _lib
    lib = _lib.lib
    not_ctx = {"b2m_last_error", "b2m_status_string", "b2m_kernel_launches", "b2m_create",
               "b2m_ReadMatrixFile", "b2m_WriteMatrixFile"}

    def zero(t):
        is_ptr = t is _lib.vp or t is ctypes.c_char_p or (hasattr(t, "_type_") and not isinstance(t._type_, str))
        return None if is_ptr else 0

    checked = 0
    for name, (_, argtypes) in _lib.SIGNATURES.items():
        if name in not_ctx:
            continue
        assert getattr(lib, name)(*[zero(t) for t in argtypes]) == _lib.ERR_ARG, name
        checked += 1
    assert checked >= 50
    assert lib.b2m_kernel_launches(None) == -1
    assert lib.b2m_last_error(None) == b"null context"
    if not torch.cuda.is_available():
        h = _lib.vp()
        assert lib.b2m_create(0, ctypes.byref(h)) == _lib.ERR_CUDA
        assert h.value is None
