"""The ITK transform files (include/fastwarp_transform_io.h) against the oracle's independent
restatement (oracle/transform_io.py), byte for byte, and the reference's own writer tests
(transform/itk_h5.rs:209-378, transform/itk_mat.rs:183-246, transform/hdf5.rs:1465-1541).

lookup3, the checksum of every metadata block, is pinned to libhdf5's through the checksums stored
in the reference's ANTs fixture (tests/golden/h5_checksums.json, made by make_h5_golden.py).
Host code only: no GPU.
"""
import json
import os
import struct

import numpy as np
import pytest

from fastwarp_b200 import FastwarpError, make_grid
from fastwarp_b200 import transform_io as T
from oracle import transform_io as O

HERE = os.path.dirname(os.path.abspath(__file__))

M = [[1.01, 0.02, 0.0], [-0.02, 0.99, 0.01], [0.0, 0.0, 1.0]]


def sample_field(size=(5, 6, 7), spacing=(2.0, 2.5, 3.0), origin=(-4.0, -5.0, -6.0),
                 direction=None):
    """itk_h5.rs:246-262: a smooth field on a 5 x 6 x 7 grid."""
    direction = np.eye(3) if direction is None else np.asarray(direction, float)
    g = make_grid(size, spacing, origin, direction)
    nx, ny, nz = size
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    p = np.stack([origin[0] + spacing[0] * x, origin[1] + spacing[1] * y,
                  origin[2] + spacing[2] * z], -1) @ direction.T
    d = np.stack([0.01 * p[..., 1] + 0.25, -0.02 * p[..., 2], 0.005 * p[..., 0] * np.sin(p[..., 1])],
                 -1).astype(np.float32)
    return g, d, O.field(size, origin, spacing, direction, d)


def test_lookup3_known_vectors_and_libhdf5_checksums():
    # lookup3.c's own self-test values (hashlittle, initval 0 and 1; the empty string)
    assert T.lookup3(b"") == O.lookup3(b"") == 0xDEADBEEF
    assert T.lookup3(b"Four score and seven years ago") == 0x17770551
    assert O.lookup3(b"Four score and seven years ago", 1) == 0xCD628161
    assert O.lookup3(b"", 0xDEADBEEF) == 0xBD5B7DDE
    blocks = json.load(open(os.path.join(HERE, "golden", "h5_checksums.json")))["blocks"]
    assert len(blocks) >= 20
    for b in blocks:
        raw = bytes.fromhex(b["bytes"])
        assert T.lookup3(raw) == b["checksum"], b["block"]
        assert O.lookup3(raw) == b["checksum"], b["block"]


@pytest.mark.parametrize("n", [0, 1, 5, 11, 12, 13, 24, 25, 100, 4097])
def test_lookup3_matches_the_oracle_at_every_tail_length(n):
    data = bytes((7 * i + 3) & 0xFF for i in range(n))
    assert T.lookup3(data) == O.lookup3(data)


def test_composite_bytes_equal_the_oracle_affine_then_field():
    g, d, of = sample_field()
    chain = [T.affine(M, [1.0, -2.0, 0.5], [3.0, 4.0, 5.0]), T.field(g, d)]
    ochain = [O.affine(M, [1.0, -2.0, 0.5], [3.0, 4.0, 5.0]), of]
    b = T.format_h5(chain)
    assert b == O.format_h5(ochain)
    # superblock v2, its checksum, end of file = the length
    assert b[:8] == b"\x89HDF\r\n\x1a\n" and b[8] == 2
    assert struct.unpack("<I", b[44:48])[0] == O.lookup3(b[:44])
    assert struct.unpack("<Q", b[28:36])[0] == len(b)
    # every object header's checksum closes it
    at = 0
    count = 0
    while (at := b.find(b"OHDR", at)) >= 0:
        flags = b[at + 5]
        width = 1 << (flags & 3)
        size = int.from_bytes(b[at + 6:at + 6 + width], "little")
        end = at + 6 + width + size
        assert struct.unpack("<I", b[end:end + 4])[0] == O.lookup3(b[at:end])
        count += 1
        at = end
    # root group + its 4 strings; TransformGroup; /0 and its type; /1 and /2 with 3 datasets
    assert count == (1 + 4) + 1 + (1 + 1) + 2 * (1 + 3)


def test_the_field_parameters_are_the_float32_values_widened():
    g, d, of = sample_field()
    b = T.format_h5([T.field(g, d)])
    wide = d.reshape(-1).astype("<f8").tobytes()
    assert b.find(wide) > 0  # contiguous, as written by the reference (F32AsF64)
    fixed = np.concatenate([[5, 6, 7], [-4.0, -5.0, -6.0], [2.0, 2.5, 3.0], np.eye(3).ravel()])
    assert b.find(fixed.astype("<f8").tobytes()) > 0  # 18 fixed parameters (grid.rs:158-169)


def test_inverse_chain_oblique_grid_and_other_os_strings():
    rot = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    g, d, of = sample_field((4, 3, 5), (1.0, 1.5, 0.5), (10.0, -3.0, 2.0), rot)
    chain = [T.field(g, -d), T.affine(np.linalg.inv(np.array(M)), [0.3, 0.2, -0.1])]
    ofm = O.field((4, 3, 5), (10.0, -3.0, 2.0), (1.0, 1.5, 0.5), rot, -d)
    ochain = [ofm, O.affine(np.linalg.inv(np.array(M)), [0.3, 0.2, -0.1])]
    assert T.format_h5(chain) == O.format_h5(ochain)
    assert T.format_h5(chain, "macos", "aarch64") == O.format_h5(ochain, "macos", "aarch64")


def test_more_than_nine_members_and_a_large_field():
    chain = [T.affine(np.eye(3), [float(i), 0.0, 0.0]) for i in range(11)]
    ochain = [O.affine(np.eye(3), [float(i), 0.0, 0.0]) for i in range(11)]
    assert T.format_h5(chain) == O.format_h5(ochain)
    # 64 x 60 x 56 voxels: 645 K values, several conversion blocks, a 4-byte chunk-size field
    g, d, of = sample_field((64, 60, 56), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0))
    assert T.format_h5([T.field(g, d)]) == O.format_h5([of])


def test_mat_file_is_193_bytes_per_affine_and_equals_the_oracle():
    a = T.affine([[0.9, 0.1, -0.05], [0.0, 1.1, 0.2], [0.03, -0.1, 1.0]], [1.0, -2.0, 3.0],
                 [-5.9, 3.1, -46.7])
    oa = O.affine([[0.9, 0.1, -0.05], [0.0, 1.1, 0.2], [0.03, -0.1, 1.0]], [1.0, -2.0, 3.0],
                  [-5.9, 3.1, -46.7])
    m = T.format_mat([a])
    assert len(m) == 193 and m == O.format_mat([oa])
    assert struct.unpack("<5I", m[:20]) == (0, 12, 1, 0, 27)
    assert m[20:47] == b"AffineTransform_double_3_3\0"
    assert np.array_equal(np.frombuffer(m[47:143], "<f8")[9:], [1.0, -2.0, 3.0])
    assert m[143 + 20:143 + 26] == b"fixed\0"
    assert T.format_mat([a, a]) == m + m


def decode_ants_mat(raw):
    """An independent decode of a MATLAB v4 file ANTs wrote for one affine transform: the
    AffineTransform_double_3_3 variable (9 matrix values row by row, then 3 translation values)
    and the `fixed` variable (the centre), each a header of five little-endian u32s, the
    variable's name with its NUL, then float64 data (samples.rs:34-67 reads the same offsets)."""
    out = {}
    at = 0
    while at < len(raw):
        mopt, mrows, ncols, imagf, namelen = struct.unpack("<5I", raw[at:at + 20])
        assert mopt == 0 and ncols == 1 and imagf == 0
        name = raw[at + 20:at + 20 + namelen - 1].decode()
        data_at = at + 20 + namelen
        out[name] = np.frombuffer(raw[data_at:data_at + 8 * mrows], "<f8")
        at = data_at + 8 * mrows
    return out


@pytest.mark.parametrize("name", ["ms0.mat", "ms20.mat"])
def test_mat_writer_reproduces_the_ants_fixtures_byte_for_byte(name):
    """The reference's ANTs-written .mat fixtures (crates/fastwarp-reg/tests/data/ms0.mat and
    ms20.mat, copied by tests/golden/make_mat_golden.py): all 193 bytes come back from the
    decoded matrix, translation and centre (tests/samples.rs:34-67)."""
    raw = open(os.path.join(HERE, "golden", "ants_" + name), "rb").read()
    assert len(raw) == 193
    v = decode_ants_mat(raw)
    assert set(v) == {"AffineTransform_double_3_3", "fixed"}
    p, c = v["AffineTransform_double_3_3"], v["fixed"]
    assert abs(np.linalg.det(p[:9].reshape(3, 3)) - 1.0) < 1e-6  # an ANTs rigid result
    out = T.format_mat([T.affine(p[:9].reshape(3, 3), p[9:], c)])
    assert out == raw
    assert O.format_mat([O.affine(p[:9].reshape(3, 3), p[9:], c)]) == raw
    if name == "ms0.mat":  # samples.rs:70-81
        assert p[0] == 0.9998442385050702 and p[1] == 0.01355877025201078
        assert p[8] == 0.9998821761749128
        assert list(p[9:]) == [-2.675791891854692, -290.9203827342067, 148.534870757413]
        assert list(c) == [-5.927373278, -3.158446675, -46.74841833]


def test_fields_in_a_mat_file_and_empty_chains_are_refused():
    g, d, _ = sample_field()
    with pytest.raises(FastwarpError, match="in a .mat file"):
        T.format_mat([T.field(g, d)])
    with pytest.raises(FastwarpError, match="empty chain"):
        T.format_h5([])
    with pytest.raises(ValueError):
        T.field(g, d[:-1])


def test_stage_outputs_are_written_whole(tmp_path):
    g, d, of = sample_field()
    fwd = [T.affine(M, [1.0, 2.0, 3.0]), T.field(g, d)]
    inv = [T.field(g, -d), T.affine(np.linalg.inv(np.array(M)), [-1.0, -2.0, -3.0])]
    total = T.affine_from_offset(M, [1.0, 2.0, 3.0], center=(3.0, 4.0, 5.0))
    paths = T.write_stage_outputs(tmp_path / "sub_", fwd, inv, total)
    assert [os.path.basename(p) for p in paths] == ["sub_Composite.h5", "sub_InverseComposite.h5",
                                                    "sub_0GenericAffine.mat"]
    assert open(paths[0], "rb").read() == T.format_h5(fwd)
    assert open(paths[1], "rb").read() == T.format_h5(inv)
    assert open(paths[2], "rb").read() == T.format_mat([total])
    assert not [p for p in os.listdir(tmp_path) if p.endswith(".tmp")]
    # the affine about a centre maps as x -> M x + offset
    t = np.array(total.c.translation[:])
    c = np.array(total.c.center[:])
    x = np.array([0.7, -1.2, 2.5])
    assert np.allclose(np.array(M) @ (x - c) + t + c, np.array(M) @ x + [1.0, 2.0, 3.0])
    with pytest.raises(FastwarpError, match="cannot open"):
        T.write_h5(tmp_path / "no_such_dir" / "x.h5", fwd)
