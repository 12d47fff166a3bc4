"""ITK transform files, restated in plain Python: the checker of the library's writers.

Test infrastructure only (like the rest of `oracle/`): tests compare the bytes the library writes
with the bytes this module builds, independently, from the same transforms.

- `lookup3`: Bob Jenkins' lookup3 `hashlittle` (public domain, 2006) with initval 0, which HDF5
  uses for its metadata checksums (transform/hdf5.rs:48-113).
- `format_h5`: the reference's HDF5 subset writer (transform/hdf5.rs:1127-1400: superblock
  version 2, version-2 object headers, compact groups with link messages, contiguous f64
  datasets, variable-length strings in one global heap collection) holding ITK's transform layout
  (transform/itk_h5.rs:108-190: HDFVersion, ITKVersion, OSName, OSVersion, TransformGroup/0 the
  composite, TransformGroup/1.. the queue).
- `format_mat`: ITK's MATLAB v4 transform file (transform/itk_mat.rs:134-165).

A transform element is ("affine", matrix 3x3, translation 3, center 3) or
("field", size 3, origin 3, spacing 3, direction 3x3 row-major, displacements AoS float32).
"""
import struct

import numpy as np

M32 = 0xFFFFFFFF


def _rot(x, k):
    return ((x << k) | (x >> (32 - k))) & M32


def lookup3(data: bytes, initval: int = 0) -> int:
    """hashlittle(data, len, initval): 12-byte blocks mixed, a 1..12-byte tail then final."""
    n = len(data)
    a = b = c = (0xDEADBEEF + n + initval) & M32
    i = 0
    while n - i > 12:
        a = (a + int.from_bytes(data[i:i + 4], "little")) & M32
        b = (b + int.from_bytes(data[i + 4:i + 8], "little")) & M32
        c = (c + int.from_bytes(data[i + 8:i + 12], "little")) & M32
        a = (a - c) & M32; a ^= _rot(c, 4); c = (c + b) & M32
        b = (b - a) & M32; b ^= _rot(a, 6); a = (a + c) & M32
        c = (c - b) & M32; c ^= _rot(b, 8); b = (b + a) & M32
        a = (a - c) & M32; a ^= _rot(c, 16); c = (c + b) & M32
        b = (b - a) & M32; b ^= _rot(a, 19); a = (a + c) & M32
        c = (c - b) & M32; c ^= _rot(b, 4); b = (b + a) & M32
        i += 12
    rest = data[i:]
    if not rest:
        return c
    tail = rest + bytes(12 - len(rest))
    a = (a + int.from_bytes(tail[0:4], "little")) & M32
    b = (b + int.from_bytes(tail[4:8], "little")) & M32
    c = (c + int.from_bytes(tail[8:12], "little")) & M32
    c ^= b; c = (c - _rot(b, 14)) & M32
    a ^= c; a = (a - _rot(c, 11)) & M32
    b ^= a; b = (b - _rot(a, 25)) & M32
    c ^= b; c = (c - _rot(b, 16)) & M32
    a ^= c; a = (a - _rot(c, 4)) & M32
    b ^= a; b = (b - _rot(a, 14)) & M32
    c ^= b; c = (c - _rot(b, 24)) & M32
    return c


UNDEF = b"\xff" * 8
F64_TYPE = bytes([0x11, 0x20, 0x3F, 0x00, 8, 0, 0, 0, 0, 0, 64, 0, 52, 11, 0, 52, 0xFF, 0x03, 0, 0])
VLEN_STR_TYPE = bytes([0x19, 0x01, 0x00, 0x00, 16, 0, 0, 0, 0x10, 0, 0, 0, 1, 0, 0, 0, 0, 0, 8, 0])


def _pad8(buf: bytearray):
    buf.extend(bytes(-len(buf) % 8))


def _object_header(messages) -> bytes:
    """Version-2 object header: signature, version, size-field width flag, chunk size, the
    messages (type, size, flags, body), lookup3 checksum."""
    total = sum(4 + len(body) for _, _, body in messages)
    flag, width = (0, 1) if total <= 0xFF else ((1, 2) if total <= 0xFFFF else (2, 4))
    out = bytearray(b"OHDR") + bytes([2, flag]) + total.to_bytes(8, "little")[:width]
    for mtype, mflags, body in messages:
        out += bytes([mtype]) + struct.pack("<H", len(body)) + bytes([mflags]) + body
    out += struct.pack("<I", lookup3(bytes(out)))
    return bytes(out)


def _dataspace(n):
    return bytes([2, 1, 1, 1]) + struct.pack("<QQ", n, n)


class _H5:
    def __init__(self, heap_addr):
        self.buf = bytearray()
        self.heap_addr = heap_addr
        self.next_string = 0

    def _dataset(self, space, dtype, raw: bytes):
        _pad8(self.buf)
        data_addr = len(self.buf)
        self.buf += raw
        _pad8(self.buf)
        at = len(self.buf)
        layout = bytes([3, 1]) + struct.pack("<QQ", data_addr, len(raw))
        self.buf += _object_header([(0x01, 1, space), (0x03, 1, dtype), (0x05, 1, bytes([3, 2])),
                                    (0x08, 0, layout)])
        return at

    def node(self, node):
        kind, value = node
        if kind == "f64":
            v = np.ascontiguousarray(value, dtype="<f8")
            return self._dataset(_dataspace(v.size), F64_TYPE, v.tobytes())
        if kind == "str":
            self.next_string += 1
            raw = struct.pack("<IQI", len(value.encode()), self.heap_addr, self.next_string)
            return self._dataset(_dataspace(1), VLEN_STR_TYPE, raw)
        return self.group(value)

    def group(self, members):
        addrs = [self.node(n) for _, n in members]
        msgs = [(0x02, 0, bytes([0, 0]) + UNDEF + UNDEF), (0x0A, 1, bytes([0, 0]))]
        for (name, _), addr in zip(members, addrs):
            nb = name.encode()
            if not 0 < len(nb) <= 0xFFFF:
                raise ValueError("bad member name length")
            body = bytes([1, 0, len(nb)]) if len(nb) <= 0xFF else bytes([1, 1]) + struct.pack("<H", len(nb))
            msgs.append((0x06, 0, body + nb + struct.pack("<Q", addr)))
        _pad8(self.buf)
        at = len(self.buf)
        self.buf += _object_header(msgs)
        return at


def _strings(members, out):
    for _, (kind, value) in members:
        if kind == "group":
            _strings(value, out)
        elif kind == "str":
            out.append(value)


def write_tree(root) -> bytes:
    """The bytes of an HDF5 file holding `root`: [(name, (kind, value))], kind in "group",
    "f64", "str"."""
    strings = []
    _strings(root, strings)
    buf = bytearray(48)
    heap_addr = 0
    if strings:
        _pad8(buf)
        heap_addr = len(buf)
        body = bytearray()
        for i, s in enumerate(strings):
            sb = s.encode()
            body += struct.pack("<HHIQ", i + 1, 1, 0, len(sb)) + sb
            _pad8(body)
        used = 16 + len(body)
        size = (max(used, 4096) + 7) // 8 * 8
        buf += b"GCOL" + bytes([1, 0, 0, 0]) + struct.pack("<Q", size) + body
        if size > used:
            buf += struct.pack("<HHIQ", 0, 0, 0, size - used)
            buf += bytes(heap_addr + size - len(buf))
    w = _H5(heap_addr)
    w.buf = buf
    root_addr = w.group(root)
    _pad8(w.buf)
    eof = len(w.buf)
    sb = bytearray(b"\x89HDF\r\n\x1a\n") + bytes([2, 8, 8, 0])
    sb += struct.pack("<Q", 0) + UNDEF + struct.pack("<QQ", eof, root_addr)
    sb += struct.pack("<I", lookup3(bytes(sb)))
    w.buf[:48] = sb
    return bytes(w.buf)


AFFINE_NAME = "AffineTransform_double_3_3"
FIELD_NAME = "DisplacementFieldTransform_double_3_3"
COMPOSITE_NAME = "CompositeTransform_double_3_3"


def affine(matrix, translation, center=(0.0, 0.0, 0.0)):
    return ("affine", np.asarray(matrix, float).reshape(3, 3), np.asarray(translation, float),
            np.asarray(center, float))


def field(size, origin, spacing, direction, data):
    return ("field", tuple(int(s) for s in size), np.asarray(origin, float),
            np.asarray(spacing, float), np.asarray(direction, float).reshape(3, 3),
            np.ascontiguousarray(data, np.float32).reshape(-1))


def _record(e):
    """(type name, fixed parameters, parameters) of an element (itk_params.rs:104-117)."""
    if e[0] == "affine":
        _, m, t, c = e
        return AFFINE_NAME, np.asarray(c, float), np.concatenate([m.reshape(-1), t])
    _, size, origin, spacing, direction, data = e
    fixed = np.concatenate([np.asarray(size, float), origin, spacing, direction.reshape(-1)])
    return FIELD_NAME, fixed, data.astype(np.float64)


def format_h5(chain, os_name="linux", os_version="x86_64") -> bytes:
    """An ITK composite transform file of `chain` (queue order)."""
    if not chain:
        raise ValueError("cannot write an empty chain")
    groups = [("0", ("group", [("TransformType", ("str", COMPOSITE_NAME))]))]
    for i, e in enumerate(chain):
        name, fixed, params = _record(e)
        groups.append((str(i + 1), ("group", [("TransformType", ("str", name)),
                                             ("TransformFixedParameters", ("f64", fixed)),
                                             ("TransformParameters", ("f64", params))])))
    root = [("HDFVersion", ("str", "1.14.0")), ("ITKVersion", ("str", "5.4.4")),
            ("OSName", ("str", os_name)), ("OSVersion", ("str", os_version)),
            ("TransformGroup", ("group", groups))]
    return write_tree(root)


def format_mat(chain) -> bytes:
    """Each affine as a `AffineTransform_double_3_3` / `fixed` pair of MATLAB v4 column vectors."""
    out = bytearray()
    for e in chain:
        if e[0] != "affine":
            raise ValueError("only affine transforms go into a .mat file")
        name, fixed, params = _record(e)
        for nm, vals in ((name, params), ("fixed", fixed)):
            v = np.ascontiguousarray(vals, "<f8")
            out += struct.pack("<5I", 0, v.size, 1, 0, len(nm) + 1) + nm.encode() + b"\0"
            out += v.tobytes()
    return bytes(out)
