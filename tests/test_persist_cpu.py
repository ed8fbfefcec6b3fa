"""Saved matrices ("RMCLS" streams of TBinaryReaderWriter, BinaryReaderWriter.pas) on the host:
the library's writer reproduces the reference's own saved fixtures byte for byte (SHA-256 recorded
in tests/golden/rmcls_matrices.json by tests/golden/make_golden.py) and its reader returns the same
numbers.  Host code only: no GPU needed."""
import hashlib
import json
import os
import struct

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "rmcls_matrices.json")


def _fixtures():
    return json.load(open(GOLDEN))


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_writer_reproduces_reference_fixture(tmp_path, idx):
    from mrmath_b200 import linalg as L
    fx = _fixtures()[idx]
    ints = fx["ints"]
    a = np.array([float.fromhex(h) for h in fx["data_hex"]]).reshape(ints["Height"], ints["Width"])
    path = str(tmp_path / "m.bin")
    L.WriteMatrixFile(path, a)
    raw = open(path, "rb").read()
    assert len(raw) == fx["size"] and hashlib.sha256(raw).hexdigest() == fx["sha256"], fx["source"]
    back, view = L.ReadMatrixFile(path)
    assert back.tobytes() == a.tobytes()
    assert view == {"sub_width": ints["SubWidth"], "sub_height": ints["SubHeight"], "offset_x": ints["OffsetX"],
                    "offset_y": ints["OffsetY"]}


def _section(typ, name, payload=b""):
    nb = name.encode()
    return struct.pack("<iBH", 7 + len(nb) + len(payload), typ, len(nb)) + nb + payload


def test_reader_takes_any_section_order_names_case_and_views(tmp_path):
    from mrmath_b200 import linalg as L
    data = np.arange(12.0).reshape(3, 4)
    body = (b"RMCLS" + struct.pack("<I", 1) + _section(10, "obj", b"MTX") + _section(5, "subwidth", struct.pack("<i", 2))
            + _section(3, "DATA", data.tobytes()) + _section(1, "Name", b"abc") + _section(5, "WIDTH", struct.pack("<i", 4))
            + _section(5, "Height", struct.pack("<i", 3)) + _section(5, "SubHeight", struct.pack("<i", 1))
            + _section(5, "OffsetX", struct.pack("<i", 1)) + _section(5, "OffsetY", struct.pack("<i", 2))
            + _section(13, ""))
    path = str(tmp_path / "v.bin")
    open(path, "wb").write(body)
    back, view = L.ReadMatrixFile(path)
    assert np.array_equal(back, data)
    assert view == {"sub_width": 2, "sub_height": 1, "offset_x": 1, "offset_y": 2}


@pytest.mark.parametrize("cls", [b"TMTX", b"B2MMTX"])
def test_reader_takes_derived_matrix_classes(tmp_path, cls):
    """TThreadedMatrix ('TMTX') and the Pascal binding's TB2MMatrix ('B2MMTX') save the same props."""
    from mrmath_b200 import linalg as L
    data = np.arange(6.0).reshape(2, 3)
    body = (b"RMCLS" + struct.pack("<I", 1) + _section(10, "obj", cls) + _section(5, "Width", struct.pack("<i", 3))
            + _section(5, "Height", struct.pack("<i", 2)) + _section(3, "data", data.tobytes()) + _section(13, ""))
    path = str(tmp_path / "d.bin")
    open(path, "wb").write(body)
    back, _ = L.ReadMatrixFile(path)
    assert np.array_equal(back, data)


def test_reader_rejects_other_streams(tmp_path):
    from mrmath_b200 import _lib, linalg as L
    bad = {
        "header": b"XMCLS" + struct.pack("<I", 1) + _section(13, ""),
        "class": b"RMCLS" + struct.pack("<I", 1) + _section(10, "obj", b"PCA") + _section(13, ""),
        "size": (b"RMCLS" + struct.pack("<I", 1) + _section(10, "obj", b"MTX")
                 + _section(5, "Width", struct.pack("<i", 3)) + _section(5, "Height", struct.pack("<i", 3))
                 + _section(3, "data", np.zeros(8).tobytes()) + _section(13, "")),
        "truncated": b"RMCLS" + struct.pack("<I", 1) + _section(10, "obj", b"MTX")[:9],
    }
    for name, raw in bad.items():
        path = str(tmp_path / f"{name}.bin")
        open(path, "wb").write(raw)
        with pytest.raises(_lib.B2MError) as ei:
            L.ReadMatrixFile(path)
        assert ei.value.status == _lib.ERR_FORMAT, name
    with pytest.raises(_lib.B2MError) as ei:
        L.ReadMatrixFile(str(tmp_path / "missing.bin"))
    assert ei.value.status == _lib.ERR_ARG
