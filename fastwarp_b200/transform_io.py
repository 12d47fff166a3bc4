"""The transform files of a registration in ITK's formats (include/fastwarp_transform_io.h).

Mirrors the reference's writers: `format_h5` / `write_h5_file` (transform/itk_h5.rs:108-200),
`format_mat` / `write_mat_file` (transform/itk_mat.rs:148-181) and `write_stage_outputs` with
the Composite layout (stages.rs:405-520: `<prefix>Composite.h5`, `<prefix>InverseComposite.h5`,
`<prefix>0GenericAffine.mat`). A chain is a list of elements in queue order, made with `affine`
and `field`.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _native as N

AFFINE, FIELD = 0, 1


class Elem:
    """One transform of a chain; keeps the arrays a field element points at alive."""

    def __init__(self, c: N.TransformElem, keep=None):
        self.c = c
        self.keep = keep


def affine(matrix, translation, center=(0.0, 0.0, 0.0)) -> Elem:
    """ITK AffineTransform: x -> M (x - c) + t + c."""
    e = N.TransformElem()
    e.kind = AFFINE
    e.matrix[:] = [float(v) for v in np.asarray(matrix, float).reshape(-1)]
    e.translation[:] = [float(v) for v in translation]
    e.center[:] = [float(v) for v in center]
    return Elem(e)


def affine_from_offset(matrix, offset, center=(0.0, 0.0, 0.0)) -> Elem:
    """The affine x -> M x + offset, written about `center` (translation = offset - c + M c)."""
    m = np.asarray(matrix, float).reshape(3, 3)
    c = np.asarray(center, float)
    return affine(m, np.asarray(offset, float) - c + m @ c, c)


def field(grid: N.Grid, data) -> Elem:
    """A displacement field on `grid`: data (nz, ny, nx, 3) or flat, float32 AoS."""
    d = np.ascontiguousarray(data, dtype=np.float32).reshape(-1)
    n = grid.size[0] * grid.size[1] * grid.size[2]
    if d.size != 3 * n:
        raise ValueError(f"field data holds {d.size} values, the grid needs {3 * n}")
    e = N.TransformElem()
    e.kind = FIELD
    e.grid = grid
    e.field = d.ctypes.data
    return Elem(e, d)


def _chain(chain):
    arr = (N.TransformElem * max(len(chain), 1))()
    for i, e in enumerate(chain):
        arr[i] = e.c
    return arr, len(chain)


def _format(fn, chain, *extra) -> bytes:
    arr, n = _chain(chain)
    size = C.c_size_t()
    N.check(fn(arr, n, *extra, None, C.c_size_t(0), C.byref(size)))
    out = (C.c_uint8 * size.value)()
    N.check(fn(arr, n, *extra, out, size, C.byref(size)))
    return bytes(out)


def format_h5(chain, os_name: str | None = None, os_version: str | None = None) -> bytes:
    """The bytes of an ITK composite transform file (OSName/OSVersion default: linux, x86_64)."""
    return _format(N.lib().fw_format_itk_h5, chain,
                   os_name.encode() if os_name else None,
                   os_version.encode() if os_version else None)


def format_mat(chain) -> bytes:
    return _format(N.lib().fw_format_itk_mat, chain)


def write_h5(path, chain) -> None:
    arr, n = _chain(chain)
    N.check(N.lib().fw_write_itk_h5(os.fsencode(path), arr, n))


def write_mat(path, chain) -> None:
    arr, n = _chain(chain)
    N.check(N.lib().fw_write_itk_mat(os.fsencode(path), arr, n))


def lookup3(data: bytes) -> int:
    return int(N.lib().fw_lookup3(data, len(data)))


def write_stage_outputs(prefix, forward, inverse, total: Elem) -> list:
    """The Composite layout of write_stage_outputs: the forward chain (the affine then the SyN
    field), the inverse chain (the inverse field then the inverse affine) and the collapsed
    affine; returns the paths written."""
    prefix = os.fspath(prefix)
    paths = [prefix + "Composite.h5", prefix + "InverseComposite.h5", prefix + "0GenericAffine.mat"]
    write_h5(paths[0], forward)
    write_h5(paths[1], inverse)
    write_mat(paths[2], [total])
    return paths
