"""Generates tests/golden/mt19937ar_kat.json from the reference's own MT19937 fixture.

Run once in a container that has the reference checked out (it is read-only input):
    python tests/golden/make_golden.py /path/to/mrmath
The fixture is the reference's Test/marsenneTwistOrig.txt (1000 genrand_int32 outputs and
1000 53-bit doubles printed with %10.8f, for init_by_array({0x123, 0x234, 0x345, 0x456}));
TestRandom.pas:249-311 compares its own output with that file byte for byte.  We keep the
parsed numbers plus the SHA-256 of the whole file, so the oracle can be pinned byte for byte
without the reference present.
"""
import hashlib
import json
import os
import sys


def main(ref_root: str) -> None:
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
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mt19937ar_kat.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
