"""Generates the golden fixtures under tests/golden/ from the reference's own test fixtures.

Run once in a container that has the reference checked out (it is read-only input):
    python tests/golden/make_golden.py /path/to/mrmath

mt19937ar_kat.json: the reference's Test/marsenneTwistOrig.txt (1000 genrand_int32 outputs and
1000 53-bit doubles printed with %10.8f, for init_by_array({0x123, 0x234, 0x345, 0x456}));
TestRandom.pas:249-311 compares its own output with that file byte for byte.  We keep the parsed
numbers plus the SHA-256 of the whole file, so the oracle can be pinned byte for byte without the
reference present.

rmcls_matrices.json: the reference's saved TDoubleMatrix objects Test/MatrixData1.txt,
Test/MatrixData2.txt (TestMatrixClass.pas:148) and Test/dyntimeWarp1.bin (TestCorr.pas:170), binary
"RMCLS" streams of TBinaryReaderWriter (BinaryReaderWriter.pas).  Parsed here by a minimal reader of
that section format (5-byte header, uint32 version, then sections {int32 length, uint8 type,
uint16 name length, name, payload} up to the end-of-stream section); we keep the sizes, the data
(as exact hex floats), the section order and the SHA-256 of each file, so the library's writer can
be checked to reproduce each file byte for byte and its reader to return the same numbers.
"""
import hashlib
import json
import os
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def mt_fixture(ref_root: str) -> None:
    path = os.path.join(ref_root, "Test", "marsenneTwistOrig.txt")
    raw = open(path, "rb").read()
    text = raw.decode("ascii")
    head_int, rest = text.split("1000 outputs of genrand_real2()")
    ints = [int(t) for t in head_int.split("genrand_int32()")[1].split()]
    reals = rest.split()
    assert len(ints) == 1000 and len(reals) == 1000
    out = {
        "source": "Test/marsenneTwistOrig.txt (used by Test/TestRandom.pas:249-311)",
        "init_key": [0x123, 0x234, 0x345, 0x456],
        "sha256": hashlib.sha256(raw).hexdigest(),
        "size": len(raw),
        "genrand_int32": ints,
        "res53_fmt_10_8f": reals,
    }
    dst = os.path.join(HERE, "mt19937ar_kat.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", dst)


def parse_rmcls(raw: bytes) -> dict:
    assert raw[:5] == b"RMCLS"
    version = struct.unpack_from("<I", raw, 5)[0]
    pos, sections, ints, data, desc = 9, [], {}, None, None
    while pos < len(raw):
        length, typ, nlen = struct.unpack_from("<iBH", raw, pos)
        name = raw[pos + 7:pos + 7 + nlen].decode("utf-8")
        payload = raw[pos + 7 + nlen:pos + length]
        sections.append([typ, name])
        if typ == 10:
            desc = payload.decode("utf-8")
        elif typ == 5:
            ints[name] = struct.unpack("<i", payload)[0]
        elif typ == 3 and name.lower() == "data":
            data = list(struct.unpack("<%dd" % (len(payload) // 8), payload))
        pos += length
        if typ == 13:
            break
    assert pos == len(raw) and desc == "MTX"
    return {"version": version, "class": desc, "sections": sections, "ints": ints,
            "data_hex": [float(x).hex() for x in data]}


def rmcls_fixtures(ref_root: str) -> None:
    out = []
    for rel, user in (("Test/MatrixData1.txt", "TestMatrixClass.pas:148"),
                      ("Test/MatrixData2.txt", "TestMatrixClass.pas:149"),
                      ("Test/dyntimeWarp1.bin", "TestCorr.pas:170")):
        raw = open(os.path.join(ref_root, rel), "rb").read()
        rec = parse_rmcls(raw)
        rec.update({"source": f"{rel} (read by {user})", "sha256": hashlib.sha256(raw).hexdigest(),
                    "size": len(raw)})
        out.append(rec)
    dst = os.path.join(HERE, "rmcls_matrices.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the mrmath checkout>")
    mt_fixture(sys.argv[1])
    rmcls_fixtures(sys.argv[1])
