"""Extracts the checksummed metadata blocks of the reference's ANTs composite transform fixture
into tests/golden/h5_checksums.json.

The fixture (WyssCenter/fastwarp, crates/fastwarp-reg/tests/data/ctest.h5) was written by
libhdf5 for ANTs: an affine then a 6 x 5 x 4 displacement field. Every metadata block of an
HDF5 file of this format ends with the Jenkins lookup3 checksum of the bytes before it; the
reference verifies them when it reads (transform/hdf5.rs:210-290, 700-770). This script records
each block's covered bytes and stored checksum -- the superblock, every version-2 object header
chunk 0 and every continuation chunk -- so the tests can pin the library's lookup3 to libhdf5's
without the fixture. Run it where the reference checkout is available:

    python tests/golden/make_h5_golden.py /path/to/fastwarp
"""
import json
import os
import struct
import sys


def blocks(d):
    out = [("superblock", 0, 44)]
    assert d[:8] == b"\x89HDF\r\n\x1a\n" and d[8] in (2, 3)
    continuations = []
    pos = 0
    while True:
        at = d.find(b"OHDR", pos)
        if at < 0:
            break
        pos = at + 4
        if d[at + 4] != 2:
            continue
        flags = d[at + 5]
        p = at + 6
        if flags & 0x20:
            p += 16
        if flags & 0x10:
            p += 4
        width = 1 << (flags & 3)
        size = int.from_bytes(d[p:p + width], "little")
        p += width
        start, end = p, p + size
        while p + 4 <= end:
            mtype, msize, mflags = d[p], struct.unpack("<H", d[p + 1:p + 3])[0], d[p + 3]
            p += 4 + (2 if flags & 0x04 else 0)
            if mtype == 0x10:
                continuations.append(struct.unpack("<QQ", d[p:p + 16]))
            p += msize
        out.append((f"OHDR@{at}", at, end - at))
        del start
    for off, length in continuations:
        assert d[off:off + 4] == b"OCHK"
        out.append((f"OCHK@{off}", off, length - 4))
    return out


def main(ref_root):
    path = os.path.join(ref_root, "crates", "fastwarp-reg", "tests", "data", "ctest.h5")
    d = open(path, "rb").read()
    rows = []
    for name, off, n in blocks(d):
        rows.append({"block": name, "bytes": d[off:off + n].hex(),
                     "checksum": struct.unpack("<I", d[off + n:off + n + 4])[0]})
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "h5_checksums.json")
    with open(out, "w") as fh:
        json.dump({"source": "crates/fastwarp-reg/tests/data/ctest.h5 (libhdf5, ANTs)",
                   "blocks": rows}, fh, indent=0)
    print(f"wrote {out}: {len(rows)} blocks")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the fastwarp checkout>")
    main(sys.argv[1])
