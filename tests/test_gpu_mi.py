"""Sampled Mattes MI of the linear stages: the CUDA level against the f64 oracle.

Tolerances of the reference's harness (crates/fastwarp-gpu/src/parity.rs:45-48): value 1e-5
relative, derivative 5e-4 relative in L2 over the parameters.
"""
import numpy as np
import pytest

import oracle as O
from cases import rot_x, rot_z
from fastwarp_b200 import CudaLinearEngine, linear_transform, make_grid

pytestmark = pytest.mark.gpu


def setup(size=(18, 17, 16), spacing=(1.3, 1.1, 1.5), origin=(-11.0, 7.0, -5.5),
          direction=None, seed=23):
    """The reference's MI known-answer case (parity.rs:101-113 Case::selftest_mi) by default."""
    direction = rot_z(0.15) @ rot_x(0.1) if direction is None else direction
    og = O.make_grid(size, spacing, origin, direction)
    g = make_grid(size, spacing, origin, direction)
    rng = np.random.default_rng(seed)
    nx, ny, nz = size
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    f = 1.0 + np.sin(0.35 * x) * np.cos(0.3 * y) + 0.6 * np.sin(0.25 * z + 0.15 * x)
    m = 1.0 + np.sin(0.35 * (x - 0.7) + 0.2) * np.cos(0.3 * (y + 0.4)) + \
        0.6 * np.sin(0.25 * (z - 0.2) + 0.15 * x) + 0.01 * rng.standard_normal(f.shape)
    f = f.astype(np.float32).astype(np.float64)
    m = m.astype(np.float32).astype(np.float64)
    pts = O.sample_points_regular(og, 0.25, 20260910)
    kept, fbin, b = O.prepare_samples(og, f, og, m, pts, 32)
    return og, g, f, m, kept, fbin, b


def transforms(center):
    base = np.array([[1.02, 0.01, 0.0], [-0.01, 0.99, 0.02], [0.0, 0.01, 1.0]])
    return {
        "euler": dict(kind="euler", parameters=[0.02, -0.03, 0.015, 0.4, -0.3, 0.2],
                      center=center),
        "euler_zyx": dict(kind="euler", parameters=[0.05, 0.02, -0.04, -0.2, 0.1, 0.3],
                          center=center, zyx=True),
        "affine_outer": dict(kind="affine", parameters=list(base.reshape(-1)) + [0.3, -0.2, 0.1],
                             center=center, outer_matrix=rot_z(0.02),
                             outer_translation=(0.1, 0.05, -0.1), outer_center=center),
    }


@pytest.mark.parametrize("tname", ["euler", "euler_zyx", "affine_outer"])
def test_value_and_derivative_match(backend, tname):
    og, g, f, m, kept, fbin, b = setup()
    center = tuple(kept.mean(0))
    kw = transforms(center)[tname]
    level = CudaLinearEngine(backend).prepare_level(g, m, kept, fbin, b)
    v, d = level.value_and_derivative(linear_transform(**kw))
    wv, wd, wn, _ = O.mi_evaluate(b, og, m, kept, fbin, O.linear_transform(**kw))
    assert abs(v - wv) <= 1e-5 * abs(wv)
    assert np.linalg.norm(d - wd) <= 5e-4 * np.linalg.norm(wd)
    assert level.num_valid() == wn
    assert abs(level.value(linear_transform(**kw)) - v) <= 1e-12 * abs(v)


def test_batched_values_equal_single_values_and_reruns_are_bit_identical(backend):
    og, g, f, m, kept, fbin, b = setup(size=(32, 30, 28), spacing=(1.0, 1.0, 1.0),
                                       origin=(0, 0, 0), direction=np.eye(3), seed=5)
    level = CudaLinearEngine(backend).prepare_level(g, m, kept, fbin, b)
    ts = [linear_transform("euler", [0.0, 0.0, 0.01 * k, 0.1 * k, 0.0, 0.0],
                           center=(15.5, 14.5, 13.5)) for k in range(6)]
    batch = level.values(ts)
    singles = [level.value(t) for t in ts]
    assert batch == singles
    a = level.value_and_derivative(ts[2])
    b2 = level.value_and_derivative(ts[2])
    assert a[0] == b2[0] and np.array_equal(a[1], b2[1])
    for t, v in zip(ts, singles):
        wv, _, _, _ = O.mi_evaluate(b, og, m, kept, fbin,
                                    O.linear_transform("euler", list(t.parameters)[:6],
                                                       center=(15.5, 14.5, 13.5)), False)
        assert abs(v - wv) <= 1e-5 * abs(wv)


def test_all_samples_outside_is_an_error(backend):
    from fastwarp_b200 import FastwarpError
    og, g, f, m, kept, fbin, b = setup()
    level = CudaLinearEngine(backend).prepare_level(g, m, kept, fbin, b)
    far = linear_transform("euler", [0, 0, 0, 500.0, 0, 0])
    with pytest.raises(FastwarpError, match="all samples map outside"):
        level.value(far)
