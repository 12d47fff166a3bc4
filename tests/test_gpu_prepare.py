"""Image preparation on the device against the oracle: isotropic resampling (register.rs:82-146),
the quantile window and intensity preprocessing (preprocess.rs:45-215), and prepare_channels_with
(register.rs:201-249).

Inputs are float32 values (what the device holds), so the reference's f64 arithmetic on them is
reproduced exactly: every comparison here is bit for bit (the oracle's f64 result rounded to
float32, as the reference's GPU backend rounds it on upload).
"""
import math

import numpy as np
import pytest

import oracle as O
from fastwarp_b200 import FastwarpError, make_grid
from fastwarp_b200.phantoms import head_pair

pytestmark = pytest.mark.gpu


def ogrid(g):
    return O.make_grid(tuple(g.size), tuple(g.spacing), tuple(g.origin),
                       np.array(g.direction[:]).reshape(3, 3))


def same(a, b):
    return np.array_equal(np.asarray(a, np.float32), np.asarray(b, np.float32), equal_nan=True)


def oblique(deg):
    t = math.radians(deg)
    return np.array([[math.cos(t), -math.sin(t), 0.0], [math.sin(t), math.cos(t), 0.0],
                     [0.0, 0.0, 1.0]])


def smooth_volume(shape, seed):
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    z, y, x = np.meshgrid(np.linspace(-1, 1, nz), np.linspace(-1, 1, ny), np.linspace(-1, 1, nx),
                          indexing="ij")
    v = 300.0 * np.exp(-(x ** 2 + 1.5 * y ** 2 + 0.7 * z ** 2)) + 40.0 * np.sin(3 * x + 2 * z)
    return (v + rng.normal(0.0, 5.0, shape)).astype(np.float32)


@pytest.fixture(scope="module")
def head(backend):
    g, fixed, _, moving, _ = head_pair()
    return g, fixed, moving


@pytest.mark.parametrize("window", [(0.0, 1.0), (0.005, 0.995), (0.25, 0.75), (0.6, 0.61)])
def test_quantile_window_and_preprocess_match_the_oracle_on_the_head_phantom(backend, head,
                                                                             window):
    g, fixed, _ = head
    img = backend.upload_image(g, fixed)
    lo, hi = window
    assert backend.quantile_window(img, lo, hi) == O.quantile_window(fixed, lo, hi)
    out = backend.preprocess(img, lo, hi).download()
    assert same(out, O.preprocess(fixed, lo, hi))


def test_preprocess_output_range_and_non_finite_voxels(backend):
    g = make_grid((47, 31, 19), (0.9, 1.1, 1.3))
    v = smooth_volume((19, 31, 47), 7)
    flat = v.reshape(-1)
    rng = np.random.default_rng(8)
    flat[rng.integers(0, flat.size, 40)] = np.nan
    flat[rng.integers(0, flat.size, 5)] = np.inf
    flat[rng.integers(0, flat.size, 5)] = -np.inf
    img = backend.upload_image(g, v)
    for lo, hi, a, b in ((0.0, 1.0, -1.0, 3.0), (0.005, 0.995, 0.0, 1.0), (0.1, 0.95, 2.0, 5.0)):
        out = backend.preprocess(img, lo, hi, a, b).download()
        assert same(out, O.preprocess(v, lo, hi, a, b))
        assert np.isnan(out[np.isnan(v)]).all()
        assert (out[v == np.inf] == b).all() and (out[v == -np.inf] == a).all()


def test_the_reference_known_answers_hold_on_the_device(backend):
    """preprocess.rs:241-287 on the device: the plain rescale, winsorised tails, the bin
    interpolation of the quantile."""
    def img(values):
        values = np.asarray(values, np.float32)
        return backend.upload_image(make_grid((values.size, 1, 1)), values.reshape(1, 1, -1))

    out = backend.preprocess(img(np.arange(1000)), 0.0, 1.0).download().ravel()
    assert out[0] == 0.0 and np.all(np.diff(out) > 0)
    assert abs(out[999] - 999.0 / (999.0 + 999.0 / 2560.0)) < 1e-6
    v = np.arange(1000, dtype=np.float32)
    v[3], v[997] = -5000.0, 9000.0
    out = backend.preprocess(img(v), 0.005, 0.995).download().ravel()
    assert out[3] == 0.0 and out[997] == 1.0
    lo, hi = backend.quantile_window(img(np.arange(2560)), 0.25, 0.75)
    assert abs(lo - 640.0) < 5.0 and abs(hi - 1920.0) < 5.0


def test_degenerate_and_non_finite_images_are_rejected(backend):
    g = make_grid((16, 8, 4))
    with pytest.raises(FastwarpError, match="degenerate intensity window"):
        backend.preprocess(backend.upload_image(g, np.full((4, 8, 16), 2.0, np.float32)), 0, 1)
    nan = np.full((4, 8, 16), np.nan, np.float32)
    nan[0, 0, :3] = np.inf
    with pytest.raises(FastwarpError, match="no finite values"):
        backend.quantile_window(backend.upload_image(g, nan), 0.0, 1.0)


@pytest.mark.parametrize("case", [
    ((21, 21, 21), (0.5, 0.5, 0.5), (0.0, 0.0, 0.0), 0.0, 1.0),
    ((37, 29, 23), (0.7, 1.3, 2.1), (-12.5, 3.25, 40.0), 0.0, 1.0),
    ((37, 29, 23), (0.7, 1.3, 2.1), (5.0, -7.0, 2.0), 25.0, 0.9),
    ((40, 33, 26), (1.2, 1.2, 1.2), (0.0, 0.0, 0.0), 10.0, 1.75),
    ((4, 1, 1), (1.5, 1.0, 1.0), (0.0, 0.0, 0.0), 0.0, 1.0),
])
def test_isotropic_resample_matches_the_oracle(backend, case):
    size, spacing, origin, deg, mm = case
    g = make_grid(size, spacing, origin, oblique(deg))
    v = smooth_volume(size[::-1], sum(size))
    out = backend.resample_isotropic(backend.upload_image(g, v), mm)
    og, ov = O.resample_isotropic(ogrid(g), v, mm)
    got = out.grid
    assert tuple(got.size) == tuple(og.size)
    assert tuple(got.spacing) == tuple(og.spacing) == (mm,) * 3
    assert tuple(got.origin) == tuple(og.origin) and tuple(got.direction) == tuple(og.direction)
    assert same(out.download(), ov)


def test_isotropic_resample_of_the_head_phantom_and_its_copy_rule(backend, head):
    g, fixed, _ = head
    img = backend.upload_image(g, fixed)
    out = backend.resample_isotropic(img, 1.5)
    og, ov = O.resample_isotropic(ogrid(g), fixed, 1.5)
    assert tuple(out.grid.size) == tuple(og.size)
    assert same(out.download(), ov)
    copy = backend.resample_isotropic(img, 1.0 + 5e-7)  # within 1e-6 mm: the image as it is
    assert tuple(copy.grid.spacing) == tuple(g.spacing) and same(copy.download(), fixed)
    for mm in (0.0, -1.0, math.nan):
        with pytest.raises(FastwarpError, match="isotropic spacing must be positive"):
            backend.resample_isotropic(img, mm)


def test_prepare_channels_composes_resampling_and_preprocessing(backend):
    fg = make_grid((30, 26, 22), (0.8, 0.8, 1.6), (1.0, 2.0, 3.0))
    mg = make_grid((28, 24, 25), (0.9, 1.0, 1.4), (-2.0, 0.0, 1.0), oblique(15.0))
    f = [smooth_volume((22, 26, 30), s) for s in (1, 2)]
    m = [smooth_volume((25, 24, 28), s) for s in (3, 4)]
    fixed = [backend.upload_image(fg, x) for x in f]
    moving = [backend.upload_image(mg, x) for x in m]
    for iso, win in ((1.0, (0.005, 0.995)), (None, None), (1.3, (0.1, 0.9))):
        channels, fraw, mraw = backend.prepare_channels(fixed, moving, iso, win)
        lo, hi = win if win is not None else (0.0, 1.0)
        for c in range(2):
            for grid, src, img, raw in ((fg, f[c], channels[c][0], fraw[c]),
                                        (mg, m[c], channels[c][1], mraw[c])):
                if iso is None:
                    rv = src
                else:
                    _, rv = O.resample_isotropic(ogrid(grid), src, iso)
                assert same(raw.download(), rv)
                assert same(img.download(), O.preprocess(rv.astype(np.float32), lo, hi))


def test_prepare_channels_rejects_what_the_reference_rejects(backend):
    g = make_grid((12, 10, 8))
    good = backend.upload_image(g, smooth_volume((8, 10, 12), 5))
    bad_v = smooth_volume((8, 10, 12), 6)
    bad_v[3, 4, 5] = np.nan
    bad = backend.upload_image(g, bad_v)
    with pytest.raises(FastwarpError, match="non-finite"):
        backend.prepare_channels([good], [bad])
    with pytest.raises(FastwarpError, match="same, non-zero number of channels"):
        backend.prepare_channels([good, good], [good])
    with pytest.raises(FastwarpError, match="winsorize must be"):
        backend.prepare_channels([good], [good], winsorize=(0.6, 0.4))
    with pytest.raises(FastwarpError, match="isotropic spacing must be positive"):
        backend.prepare_channels([good], [good], iso_mm=-2.0)
