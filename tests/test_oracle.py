"""Pins the CPU oracle (oracle/) against the reference's own known answers.

Each test restates a unit test of WyssCenter/fastwarp (crate fastwarp-reg, paths below relative to
crates/fastwarp-reg/src) or checks the ITK 5.4.5 golden fixtures the reference ships
(crates/fastwarp-reg/tests/data/mattes, repacked into tests/golden/mattes_itk.npz).
"""
import math
import os

import numpy as np
import pytest

import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "mattes_itk.npz")


def cube(n, spacing=1.0):
    return O.make_grid((n, n, n), (spacing,) * 3)


def noise(g, seed, mod=997):
    n = g.size[0] * g.size[1] * g.size[2]
    i = np.arange(n, dtype=np.uint64)
    v = (((i + np.uint64(seed)) * np.uint64(2654435761)) % np.uint64(mod)).astype(np.float64) / mod
    return v.reshape(O.grid_shape(g))


# ---- sampling.rs:243-266 ---------------------------------------------------------------------

def test_mt19937_matches_the_published_reference_outputs():
    first = O.mt19937(5489, 10)
    assert list(first) == [3499211612, 581869302, 3890346734, 3586334585, 545404204,
                           4161255391, 3922919429, 949333985, 2715962298, 1323567403]
    assert O.mt19937(5489, 10000)[-1] == 4123659995


def test_regular_sampling_takes_every_stride_th_voxel_jittered_by_a_third_of_the_spacing():
    g = O.make_grid((10, 9, 8), (2.0, 1.0, 1.5))
    pts = O.sample_points_regular(g, 0.25, 20260910)
    assert pts.shape == (math.ceil(720 / 4), 3)
    # voxel q*4 in raster order, displaced by N(0,1)*spacing/3 (bounded by ~5 sigma)
    for q in (0, 7, 100):
        flat = 4 * q
        idx = (flat % 10, (flat // 10) % 9, flat // 90)
        base = O.index_to_point(g, idx)
        assert np.all(np.abs(pts[q] - base) < 5.0 * np.array([2.0, 1.0, 1.5]) / 3.0)


# ---- field_ops.rs:655-716 (Gaussian operator) -------------------------------------------------

def series_i(n, t):
    s, term = 0.0, (t / 2.0) ** n
    for k in range(n):
        term /= k + 1
    for k in range(60):
        s += term
        term *= (t / 2.0) ** 2 / ((k + 1) * (k + 1 + n))
    return s


@pytest.mark.parametrize("variance", [0.5, 1.0, 3.0, 8.0])
def test_operator_taps_match_the_bessel_series_definition(variance):
    taps = O.gaussian_taps(variance)
    r = len(taps) // 2
    assert len(taps) == 2 * r + 1
    assert abs(taps.sum() - 1.0) < 1e-12
    assert np.allclose(taps, taps[::-1], atol=1e-15)
    raw = [math.exp(-variance) * series_i(n, variance) for n in range(r + 1)]
    one_sided = raw[0] + 2 * sum(raw[1:])
    assert one_sided >= 0.999 - 1e-5
    assert raw[0] + 2 * sum(raw[1:r]) < 0.999 + 1e-5
    for n in range(r + 1):
        assert abs(taps[r + n] - raw[n] / one_sided) < 5e-6


def test_variance_three_kernel_has_radius_six_and_the_expected_centre():
    taps = O.gaussian_taps(3.0)
    assert len(taps) // 2 == 6
    assert abs(taps[6] - 0.2433) < 5e-4
    short = O.gaussian_taps(3.0, max_width=3)
    assert len(short) // 2 == 3 and abs(short.sum() - 1.0) < 1e-12


# ---- field_ops.rs:718-755 (smoothing) -------------------------------------------------------

def test_smoothing_a_delta_returns_the_kernel_and_pins_the_boundary():
    g = cube(21)
    f = np.zeros((21, 21, 21, 3))
    f[10, 10, 10, 0] = 1.0
    s = O.smooth_field(g, f, 3.0)
    taps = O.gaussian_taps(3.0, 0.001, 21)
    r = len(taps) // 2
    for t in range(len(taps)):
        assert abs(s[10, 10, 10 + t - r, 0] - taps[t] * taps[r] * taps[r]) < 1e-14
    faces = np.ones((21, 21, 21), bool)
    faces[1:-1, 1:-1, 1:-1] = False
    assert np.all(s[faces] == 0.0)


def test_smoothing_preserves_a_constant_inside_and_blends_below_half_variance():
    g = cube(15)
    f = np.broadcast_to(np.array([2.0, -1.0, 0.5]), (15, 15, 15, 3)).copy()
    assert np.allclose(O.smooth_field(g, f, 3.0)[7, 7, 7], [2.0, -1.0, 0.5], atol=1e-12)
    assert np.allclose(O.smooth_field(g, f, 0.25)[7, 7, 7], [2.0, -1.0, 0.5], atol=1e-12)
    assert np.array_equal(O.smooth_field(g, f, 0.0), f)


def test_max_scaled_norm_propagates_a_non_finite_voxel():
    g = O.make_grid((5, 4, 3))
    f = np.zeros((3, 4, 5, 3))
    f[..., 0] = np.arange(5)[None, None, :]
    assert O.max_scaled_norm(g, f) == 4.0
    f.reshape(-1, 3)[17, 0] = np.nan
    assert math.isnan(O.max_scaled_norm(g, f))


# ---- field_ops.rs:757-861 (compose, invert, resample) -----------------------------------------

def test_compose_with_constants_adds_them_and_outside_the_buffer_the_update_is_zero():
    g = cube(8, 2.0)
    u = np.broadcast_to([1.0, 2.0, 3.0], (8, 8, 8, 3)).copy()
    w = np.broadcast_to([0.5, 0.0, -0.5], (8, 8, 8, 3)).copy()
    assert np.all(O.compose(g, u, w) == np.array([1.5, 2.0, 2.5]))
    far = np.broadcast_to([100.0, 0.0, 0.0], (8, 8, 8, 3)).copy()
    assert np.all(O.compose(g, u, far) == np.array([100.0, 0.0, 0.0]))


def test_compose_follows_the_warping_field_for_a_linear_displacement():
    g = cube(10)
    x = np.arange(10, dtype=float)
    u = np.zeros((10, 10, 10, 3))
    u[..., 0] = 0.1 * x[None, None, :]
    w = np.zeros_like(u)
    w[..., 0] = 1.0
    c = O.compose(g, u, w)
    assert abs(c[4, 4, 3, 0] - (1.0 + 0.4)) < 1e-12


def sine_field(n, spacing, amp):
    s = spacing
    idx = np.arange(n, dtype=float)
    p = idx * s
    x = p / ((n - 1) * s)
    w = (np.sin(np.pi * x)[None, None, :] * np.sin(np.pi * x)[None, :, None] *
         np.sin(np.pi * x)[:, None, None])
    return np.stack([amp * w, -0.7 * amp * w, 0.5 * amp * w], axis=-1)


def test_inverse_of_a_smooth_field_composes_to_identity_within_the_filter_tolerance():
    g = cube(24, 1.5)
    u = sine_field(24, 1.5, 2.0)
    inv, (it, mean, mx) = O.invert(g, u)
    assert 2 <= it <= 20
    assert mx <= 0.1 or mean <= 0.001 or it == 20
    res = O.compose(g, u, inv)
    norms = np.sqrt(((res / 1.5) ** 2).sum(-1))
    assert norms[1:-1, 1:-1, 1:-1].max() < 0.1
    faces = np.ones((24, 24, 24), bool)
    faces[1:-1, 1:-1, 1:-1] = False
    assert np.all(inv[faces] == 0.0)
    again, (it2, _, mx2) = O.invert(g, u, inv)
    assert it2 == 1 and mx2 < 0.1
    assert np.abs(again[..., 0] - inv[..., 0]).max() < 0.05


def test_inversion_stops_at_the_iteration_limit_and_reports_the_pre_update_error():
    g = cube(12)
    u = sine_field(12, 1.0, 3.0)
    _, (it, _, mx3) = O.invert(g, u, params=(3, 0.0, 0.0, True))
    assert it == 3
    _, (it1, _, mx1) = O.invert(g, u, params=(1, 0.0, 0.0, True))
    assert it1 == 1 and mx1 > mx3
    zero = np.zeros((12, 12, 12, 3))
    inv, (itz, _, _) = O.invert(g, zero)
    assert itz == 1 and np.all(inv == 0.0)


def test_resampling_reproduces_a_linear_field_and_is_zero_outside_the_old_buffer():
    coarse = cube(8, 2.0)
    p = np.arange(8) * 2.0
    f = np.zeros((8, 8, 8, 3))
    f[..., 0] = 0.1 * p[None, None, :] + 1.0
    f[..., 1] = 0.2 * p[None, :, None]
    f[..., 2] = -0.05 * p[:, None, None]
    fine = cube(13)
    r = O.resample_field(coarse, f, fine)
    assert abs(r[7, 6, 5, 0] - (0.1 * 5 + 1.0)) < 1e-12
    assert abs(r[7, 6, 5, 1] - 0.2 * 6) < 1e-12
    wide = O.make_grid((8, 8, 8), (2.0,) * 3, (-20.0, 0.0, 0.0))
    assert np.all(O.resample_field(coarse, f, wide)[3, 3, 0] == 0.0)
    assert np.array_equal(O.resample_field(coarse, f, coarse), f)


# ---- cpu/mod.rs:619-708 (warp, CC) ------------------------------------------------------------

def ramp(g):
    z, y, x = np.meshgrid(*[np.arange(s) for s in O.grid_shape(g)], indexing="ij")
    return 2.0 * x + 5.0 * y - z


def test_warp_through_a_zero_field_is_the_identity_and_translates_with_an_affine():
    g = O.make_grid((8, 7, 6), (1.5, 1.5, 2.0), (-3.0, 2.0, 1.0))
    v = ramp(g)
    zero = np.zeros(O.grid_shape(g) + (3,))
    assert np.allclose(O.warp(g, v, g, zero), v, atol=1e-12)
    moved = O.warp(g, v, g, zero, affine=O.make_affine(offset=(3.0, 0.0, 0.0)))
    assert abs(moved[2, 3, 2] - (2.0 * 4.0 + 15.0 - 2.0)) < 1e-12
    assert moved[2, 3, 7] == 0.0


def test_warp_applies_the_field_before_the_affine_and_pre_between():
    g = O.make_grid((8, 7, 6), (1.5, 1.5, 2.0), (-3.0, 2.0, 1.0))
    v = ramp(g)
    fld = np.broadcast_to([1.5, 0.0, 0.0], O.grid_shape(g) + (3,)).copy()
    pre_grid = O.make_grid((4, 7, 6), (1.5, 1.5, 2.0), (-3.0, 2.0, 1.0))
    pre = np.broadcast_to([0.0, 1.5, 0.0], O.grid_shape(pre_grid) + (3,)).copy()
    aff = O.make_affine(np.diag([0.5, 1.0, 1.0]))
    out = O.warp(g, v, g, fld, pre_grid, pre, aff)
    ones = np.ones(O.grid_shape(g))
    mask = O.warp_mask(g, ones, g, fld, pre_grid, pre, aff)
    for i, in_pre in [(0, True), (6, False)]:
        x = O.index_to_point(g, (i, 2, 2))
        q = x + [1.5, 0, 0]
        assert O.point_to_index(pre_grid, q)[0] < 3.5 if in_pre else True
        r = q + ([0, 1.5, 0] if in_pre else [0, 0, 0])
        s = np.array([0.5 * r[0], r[1], r[2]])
        c = O.point_to_index(g, s)
        inside = all(-0.5 <= c[a] < [8, 7, 6][a] - 0.5 for a in range(3))
        want = O.warp(g, v, g, np.zeros_like(fld), affine=O.make_affine(offset=s - x))[2, 2, i]
        assert abs(out[2, 2, i] - (want if inside else 0.0)) < 1e-12
        near = all(0 <= math.floor(c[a] + 0.5) < [8, 7, 6][a] for a in range(3))
        assert mask[2, 2, i] == float(near)


def test_cc_of_an_image_with_itself_is_minus_one_with_zero_derivative():
    g = cube(9)
    v = noise(g, 0)
    val, d, _, _, nv = O.cc(g, v, v, 2)
    assert abs(val + 1.0) < 1e-12 and np.abs(d).max() < 1e-9 and nv == 729


def brute(f, m, valid, r, k, j, i):
    sl = tuple(slice(max(c - r, 0), c + r + 1) for c in (k, j, i))
    ok = valid[sl]
    a, b = f[sl][ok], m[sl][ok]
    n = ok.sum()
    ffv = (a * a).sum() - a.sum() ** 2 / n
    mmv = (b * b).sum() - b.sum() ** 2 / n
    fmv = (a * b).sum() - a.sum() * b.sum() / n
    return fmv * fmv / (ffv * mmv) if abs(ffv * mmv) > np.finfo(float).eps else 1.0


def test_window_statistics_match_a_brute_force_neighbourhood_with_invalid_voxels():
    g = cube(9)
    f, m = noise(g, 3), noise(g, 11)
    k, j, i = np.meshgrid(np.arange(9), np.arange(9), np.arange(9), indexing="ij")
    valid = ~((np.sqrt((i - 4.0) ** 2 + (j - 3.5) ** 2 + (k - 5.0) ** 2) < 2.6) | (i == 0) |
              ((j == 8) & (k > 4)))
    val, d, lcc, coeff, nv = O.cc(g, f, m, 2, valid=valid.astype(float) * 3.0)
    assert nv == valid.sum()
    total = 0.0
    for kk, jj, ii in zip(*np.nonzero(valid)):
        want = brute(f, m, valid, 2, kk, jj, ii)
        assert abs(lcc[kk, jj, ii] - want) < 1e-9
        total += want
    assert abs(val + total / nv) < 1e-12
    assert np.all(lcc[~valid] == 0.0) and np.all(coeff[~valid] == 0.0)
    with pytest.raises(O.OracleError, match="no voxel of the registration level"):
        O.cc(g, f, m, 2, valid=np.zeros((9, 9, 9)))


def test_cc_coefficient_is_the_derivative_of_the_local_cc_wrt_the_centre_voxel():
    g = cube(9)
    f, m = noise(g, 2, 1000), noise(g, 9, 1000)
    _, _, _, coeff, _ = O.cc(g, f, m, 2)
    for (i, j, k) in [(4, 4, 4), (0, 0, 0), (8, 3, 5), (1, 7, 2)]:
        h = 1e-6
        up, dn = m.copy(), m.copy()
        up[k, j, i] += h
        dn[k, j, i] -= h
        fd = (O.cc(g, f, up, 2)[2][k, j, i] - O.cc(g, f, dn, 2)[2][k, j, i]) / (2 * h)
        assert abs(fd - coeff[k, j, i]) < 1e-5 * (1 + abs(fd))


def test_cc_is_invariant_to_affine_intensity_changes_of_either_image():
    g = cube(10)
    f = noise(g, 5, 1000)
    z, y, x = np.meshgrid(*[np.arange(10.0)] * 3, indexing="ij")
    m = 1 + np.sin(0.45 * (x - 0.3)) * np.cos(0.35 * (y - 0.2)) + 0.5 * np.sin(0.3 * (z - 0.1) + 0.2 * x)
    base = O.cc(g, f, m, 3)
    a = O.cc(g, f, -2.5 * m + 7.0, 3)
    b = O.cc(g, 4.0 * f - 1.0, m, 3)
    for other in (a, b):
        assert abs(base[0] - other[0]) < 1e-9
        assert np.abs(base[2] - other[2]).max() < 1e-9
    assert np.abs(base[1] - a[1]).max() < 1e-8


# ---- interp.rs:143-168 -------------------------------------------------------------------------

def test_linear_interpolation_clamps_the_half_voxel_border():
    g = O.make_grid((5, 4, 3), (2.0, 1.5, 1.0), (1.0, -2.0, 3.0))
    z, y, x = np.meshgrid(np.arange(3.0), np.arange(4.0), np.arange(5.0), indexing="ij")
    v = 2 * x - 3 * y + 0.5 * z
    zero = np.zeros((3, 4, 5, 3))
    # warp by a constant physical shift of -0.4 voxels in x reads the edge voxel at i=0
    shifted = O.warp(g, v, g, zero, affine=O.make_affine(offset=(-0.4 * 2.0, 0.0, 0.0)))
    assert shifted[0, 0, 0] == 0.0  # c = -0.4: base clamped, weight zero -> v[0] = 0
    past = O.warp(g, v, g, zero, affine=O.make_affine(offset=(-0.6 * 2.0, 0.0, 0.0)))
    assert past[0, 0, 0] == 0.0 and past[1, 1, 1] == pytest.approx(v[1, 1, 1] - 2 * 0.6)


# ---- convergence.rs:129-214 --------------------------------------------------------------------

def test_convergence_monitor_matches_the_closed_form_of_the_two_point_fit():
    vals = [9.0, 8.5, 8.2, 8.0, 7.9, 7.85, 7.82, 7.80, 7.79, 7.785]
    total = sum(vals)
    eps = 1e-4
    d0 = d1 = o0 = o1 = 0.0
    for n, v in enumerate(vals):
        p = n / 9.0
        if abs(p - 1.0) <= eps:
            p = 1.0 - eps
        t0, t1 = 1.0 - p, p
        s = t0 * t0 + t1 * t1
        yv = v / total
        o0 += t0 * t0
        o1 += t1 * t1
        d0 += yv * t0 ** 3 / s
        d1 += yv * t1 ** 3 / s
    got = O.convergence_value(vals, 10, total)
    assert abs(got - (d0 / o0 - d1 / o1)) < 1e-14 and got > 0.0
    assert O.convergence_value(vals[:9], 10, total) == np.finfo(np.float64).max
    flat = O.convergence_value([-0.5] * 10, 10, 5.0)
    assert abs(flat) < 1e-4


# ---- metric/mi.rs:819-1157 ---------------------------------------------------------------------

def test_cubic_bspline_kernels_partition_unity_and_the_derivative_matches_fd():
    for t in [0.0, 0.1, 0.37, 0.5, 0.99]:
        assert abs(sum(O.bspline3(k - t) for k in range(-1, 3)) - 1.0) < 1e-12
        assert abs(sum(O.bspline3_derivative(k - t) for k in range(-1, 3))) < 1e-12
    for u in [-1.7, -1.2, -0.6, -0.1, 0.2, 0.9, 1.4, 1.9]:
        h = 1e-6
        fd = (O.bspline3(u + h) - O.bspline3(u - h)) / (2 * h)
        assert abs(fd - O.bspline3_derivative(u)) < 1e-6
    assert O.bspline3(2.0) == 0.0 and abs(O.bspline3(0.0) - 4.0 / 6.0) < 1e-15


def smooth_vol(n, shift, phase):
    z, y, x = np.meshgrid(*[np.arange(n, dtype=float)] * 3, indexing="ij")
    x, y, z = x - shift[0], y - shift[1], z - shift[2]
    return 1.0 + np.sin(0.35 * x + phase) * np.cos(0.3 * y) + 0.6 * np.sin(0.25 * z + 0.15 * x)


def mi_setup(n=14, shift=(0.7, -0.4, 0.2), phase=0.2, interior=None):
    g = cube(n)
    f = smooth_vol(n, (0, 0, 0), 0.0)
    m = smooth_vol(n, shift, phase)
    pts = O.sample_points_regular(g, 0.25, 20260910)
    if interior is not None:
        pts = pts[np.all((pts >= interior[0]) & (pts <= interior[1]), axis=1)]
    kept, fbin, b = O.prepare_samples(g, f, g, m, pts, 32)
    return g, f, m, kept, fbin, b


def test_binning_follows_the_itk_padding_rule():
    g, f, m, kept, fbin, b = mi_setup(12, (0.5, 0, 0), 0.3)
    assert abs(b.fixed_bin_size - (b.fixed_max - b.fixed_min) / 28.0) < 1e-15
    assert abs(b.moving_normalized_min - (b.moving_min / b.moving_bin_size - 2.0)) < 1e-12
    assert fbin.min() >= 2 and fbin.max() <= 29


def test_pdf_is_normalised_and_the_value_is_minus_the_mutual_information():
    g, f, m, kept, fbin, b = mi_setup()
    t = O.linear_transform("euler")
    val, _, nv, joint = O.mi_evaluate(b, g, m, kept, fbin, t, want_derivative=False)
    assert abs(joint.sum() - 1.0) < 1e-12
    pf, pm = joint.sum(1), joint.sum(0)
    nz = joint > 1e-12
    mi = (joint[nz] * np.log(joint[nz] / np.outer(pf, pm)[nz])).sum()
    assert abs(val + mi) < 1e-9 and mi > 0 and 0 < nv <= len(kept)


@pytest.mark.parametrize("kind", ["euler", "affine"])
def test_mi_derivative_matches_central_differences_of_the_value(kind):
    g, f, m, kept, fbin, b = mi_setup(26, (1.1, -0.8, 0.6), 0.0, interior=(6.0, 19.0))
    if kind == "euler":
        t = O.linear_transform("euler", [0.01, -0.02, 0.015, 0.4, -0.3, 0.2], center=(13, 13, 13))
    else:
        base = np.array([[1.0, 0.01, 0.0], [-0.01, 1.0, 0.0], [0.0, 0.0, 1.0]])
        t = O.linear_transform("affine", list(base.reshape(-1)) + [0.3, -0.2, 0.1],
                               center=(13, 13, 13), outer_translation=(0.1, 0.05, -0.1))
    val, der, nv, _ = O.mi_evaluate(b, g, m, kept, fbin, t)
    params = list(t.parameters)[:len(der)]
    fd = []
    for k in range(len(params)):
        h = 1e-4 if (k < 3 and len(params) == 6) else 1e-3
        up, dn = list(params), list(params)
        up[k] += h
        dn[k] -= h
        tu = O.linear_transform(kind, up, center=(13, 13, 13),
                                outer_translation=tuple(t.outer_translation))
        td = O.linear_transform(kind, dn, center=(13, 13, 13),
                                outer_translation=tuple(t.outer_translation))
        vu, _, nu, _ = O.mi_evaluate(b, g, m, kept, fbin, tu, False)
        vd, _, nd, _ = O.mi_evaluate(b, g, m, kept, fbin, td, False)
        assert nu == nv and nd == nv
        fd.append(-(vu - vd) / (2 * h))
    fd = np.array(fd)
    assert np.abs(fd).max() > 1e-4
    assert np.abs(der - fd).max() <= 0.08 * np.abs(fd).max()


def test_euler_jacobian_matches_finite_differences_in_both_orders():
    p = np.array([12.0, -7.0, 31.0])
    for zyx in (False, True):
        params = [0.21, -0.17, 0.33, 1.0, -2.0, 0.5]
        t = O.linear_transform("euler", params, center=(3.0, 4.0, -5.0), zyx=zyx)
        cols = O.linear_jacobian(t, p)
        for k in range(6):
            h = 1e-6
            up, dn = list(params), list(params)
            up[k] += h
            dn[k] -= h
            mu, ou = O.linear_map(O.linear_transform("euler", up, center=(3, 4, -5), zyx=zyx))
            md, od = O.linear_map(O.linear_transform("euler", dn, center=(3, 4, -5), zyx=zyx))
            fd = ((mu @ p + ou) - (md @ p + od)) / (2 * h)
            assert np.abs(cols[k] - fd).max() < 1e-6


# ---- ITK 5.4.5 golden fixtures (crates/fastwarp-reg/tests/mattes_itk.rs:99-200) ---------------

FIXTURES = ["oblique_b12", "oblique_b32", "oblique_b32_masked", "virtual_b32",
            "virtual_b32_masked", "virtual_b32_masked_swapped"]


@pytest.mark.parametrize("name", FIXTURES)
def test_dense_mattes_matches_itk(name):
    z = np.load(GOLDEN)

    def grid(role):
        return O.make_grid(z[f"{name}/{role}_size"].astype(int), z[f"{name}/{role}_spacing"],
                           z[f"{name}/{role}_origin"], z[f"{name}/{role}_direction"].reshape(3, 3))

    fg, mg = grid("fixed"), grid("moving")
    fld = z[f"{name}/field"].astype(np.float32).astype(np.float64)
    fm = z[f"{name}/fixed_mask"] if f"{name}/fixed_mask" in z.files else None
    mm = z[f"{name}/moving_mask"] if f"{name}/moving_mask" in z.files else None
    v, nv, d = O.mi_dense(fg, z[f"{name}/fixed"], mg, z[f"{name}/moving"], fld,
                          int(z[f"{name}/bins"][0]), fg if fm is not None else None, fm,
                          mg if mm is not None else None, mm)
    want = z[f"{name}/value"][0]
    wd = z[f"{name}/derivative"].reshape(-1, 3)
    assert nv == int(z[f"{name}/valid"][0])
    assert abs(v - want) <= 1e-12 * abs(want)
    d = d.reshape(-1, 3)
    assert np.array_equal(np.all(d == 0, axis=1), np.all(wd == 0, axis=1))
    assert np.abs(d - wd).max() <= 1e-10 * np.abs(wd).max()


# ---- pyramid.rs (shrink factors and grids) -----------------------------------------------------

def test_shrink_factors_go_to_the_finest_axis_and_grids_keep_their_centre():
    assert O.shrink_factors(4, (1.0, 1.0, 1.0)) == (4, 4, 4)
    assert O.shrink_factors(4, (1.0, 2.0, 1.0)) == (4, 2, 4)
    g = O.make_grid((193, 229, 193), (1.0, 1.0, 1.0), (-96.0, -132.0, -78.0))
    s = O.shrink_grid(g, (4, 4, 4))
    assert tuple(s.size) == (48, 57, 48) and tuple(s.spacing) == (4.0, 4.0, 4.0)
    c_in = O.index_to_point(g, [(n - 1) / 2 for n in (193, 229, 193)])
    c_out = O.index_to_point(s, [(n - 1) / 2 for n in (48, 57, 48)])
    assert np.allclose(c_in, c_out, atol=1e-12)


def test_recursive_gaussian_keeps_a_constant_and_approximates_a_gaussian():
    from scipy.ndimage import gaussian_filter
    g = O.make_grid((40, 36, 32))
    const = np.full((32, 36, 40), 3.0)
    assert np.allclose(O.smooth_recursive(g, const, (2.0, 2.0, 2.0)), 3.0, atol=1e-9)
    rng = np.random.default_rng(0)
    img = gaussian_filter(rng.standard_normal((32, 36, 40)), 1.0)
    a = O.smooth_recursive(g, img, (2.0, 2.0, 2.0))
    b = gaussian_filter(img, 2.0, mode="nearest")
    inner = (slice(8, -8),) * 3
    assert np.abs(a[inner] - b[inner]).max() < 0.02 * np.abs(b[inner]).max()


# ---- syn_phantom.rs:383-512 (the loop recovers a known smooth deformation) ---------------------

def test_syn_loop_reduces_the_cc_energy_on_a_blob_pair():
    rng = np.random.default_rng(3)
    n = 24
    g = cube(n)
    z, y, x = np.meshgrid(*[np.arange(n, dtype=float)] * 3, indexing="ij")
    f = np.exp(-(((x - 11) / 5) ** 2 + ((y - 12) / 4) ** 2 + ((z - 12) / 6) ** 2)) + \
        0.6 * np.exp(-(((x - 16) / 3) ** 2 + ((y - 8) / 3) ** 2 + ((z - 14) / 3) ** 2))
    m = np.exp(-(((x - 12) / 5) ** 2 + ((y - 11.5) / 4) ** 2 + ((z - 12) / 6) ** 2)) + \
        0.6 * np.exp(-(((x - 17) / 3) ** 2 + ((y - 8.5) / 3) ** 2 + ((z - 14) / 3) ** 2))
    r = O.syn_recipe(gradient_step=0.25, update_variance=3.0, cc_radius=2, iterations=(15,),
                     shrink=(1,), sigmas=(0.0,), convergence_threshold=-1.0)
    warp, inv, recs, last = O.syn_run(r, g, [f], g, [m])
    assert len(recs) == 15
    assert recs[-1].energy < recs[0].energy - 0.003
    assert all(s.iterations >= 1 for rec in recs for s in rec.inversions)


# ---- masked SyN (syn.rs:496-580; syn.rs:1239-1300; syn_phantom.rs:290-380) ---------------------

def _cavity_pair(n=24):
    z, y, x = np.meshgrid(*[np.arange(n, dtype=float)] * 3, indexing="ij")
    f = np.exp(-(((x - 11) / 5) ** 2 + ((y - 12) / 4) ** 2 + ((z - 12) / 6) ** 2)) + \
        0.6 * np.exp(-(((x - 16) / 3) ** 2 + ((y - 8) / 3) ** 2 + ((z - 14) / 3) ** 2))
    m = np.exp(-(((x - 12) / 5) ** 2 + ((y - 11.5) / 4) ** 2 + ((z - 12) / 6) ** 2)) + \
        0.6 * np.exp(-(((x - 17) / 3) ** 2 + ((y - 8.5) / 3) ** 2 + ((z - 14) / 3) ** 2))
    return f, m, (x, y, z)


def test_masks_of_ones_leave_the_syn_run_unchanged():
    n = 20
    g = cube(n)
    f, m, _ = _cavity_pair(n)
    r = O.syn_recipe(gradient_step=0.25, update_variance=3.0, cc_radius=2, iterations=(4, 3),
                     shrink=(2, 1), sigmas=(1.0, 0.0), convergence_threshold=-1.0)
    w0, i0, r0, _ = O.syn_run(r, g, [f], g, [m])
    ones = np.ones((n, n, n))
    mg = O.make_grid((n + 4,) * 3, (1.0,) * 3, (-2.0,) * 3)
    w1, i1, r1, _ = O.syn_run(r, g, [f], g, [m], masks=dict(
        fixed_grid=g, fixed=ones, moving_grid=mg, moving=np.ones((n + 4,) * 3)))
    assert np.array_equal(w0, w1) and np.array_equal(i0, i1)
    assert [a.energy for a in r0] == [b.energy for b in r1]


def test_a_moving_mask_keeps_a_cavity_from_driving_the_deformation():
    n = 24
    g = cube(n)
    f, m, (x, y, z) = _cavity_pair(n)
    centre = (8.0, 15.0, 12.0)
    inside = (x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2 < 4.0 ** 2
    lesioned = np.where(inside, 0.9, m)
    # the mask on its own coarser grid: 0 in a ball a little bigger than the cavity
    mg = O.make_grid((17, 17, 17), (1.5, 1.5, 1.5), (0.0, 0.0, 0.0))
    mz, my, mx = np.meshgrid(*[np.arange(17) * 1.5] * 3, indexing="ij")
    keep = ((mx - centre[0]) ** 2 + (my - centre[1]) ** 2 + (mz - centre[2]) ** 2 >= 5.5 ** 2)
    r = O.syn_recipe(gradient_step=0.25, update_variance=3.0, cc_radius=2, iterations=(12,),
                     shrink=(1,), sigmas=(0.0,), convergence_threshold=-1.0)
    clean, _, _, _ = O.syn_run(r, g, [f], g, [m])
    unmasked, _, _, _ = O.syn_run(r, g, [f], g, [lesioned])
    masked, _, _, _ = O.syn_run(r, g, [f], g, [lesioned],
                                masks=dict(moving_grid=mg, moving=keep.astype(float)))
    near = inside
    dev_u = np.sqrt(((unmasked - clean) ** 2).sum(-1))[near].mean()
    dev_m = np.sqrt(((masked - clean) ** 2).sum(-1))[near].mean()
    assert dev_u > 0.05, dev_u
    assert dev_m < 0.5 * dev_u, (dev_m, dev_u)


def test_an_all_zero_mask_is_refused():
    n = 12
    g = cube(n)
    f, m, _ = _cavity_pair(n)
    r = O.syn_recipe(gradient_step=0.25, update_variance=3.0, cc_radius=2, iterations=(2,),
                     shrink=(1,), sigmas=(0.0,), convergence_threshold=-1.0)
    with pytest.raises(RuntimeError, match="fixed mask has no voxel inside"):
        O.syn_run(r, g, [f], g, [m], masks=dict(fixed_grid=g, fixed=np.zeros((n, n, n))))


def test_a_mattes_channel_syn_loop_reduces_its_energy():
    """SynMetric::Mattes channels (syn.rs:301-335): the dense MI pair drives the loop."""
    n = 24
    g = cube(n)
    f, m, _ = _cavity_pair(n)
    r = O.syn_recipe(gradient_step=0.1, update_variance=3.0, cc_radius=2, iterations=(12,),
                     shrink=(1,), sigmas=(0.0,), convergence_threshold=-1.0,
                     metrics=["mattes"], mi_bins=32)
    warp, inv, recs, _ = O.syn_run(r, g, [f], g, [m])
    assert len(recs) == 12
    assert recs[-1].energy < recs[0].energy - 0.1  # -MI: lower is better
    assert np.isfinite(warp).all() and np.abs(warp).max() > 0.1


def test_a_cc_and_a_mattes_channel_combine():
    n = 20
    g = cube(n)
    f, m, _ = _cavity_pair(n)
    r = O.syn_recipe(gradient_step=0.25, update_variance=3.0, cc_radius=2, iterations=(4,),
                     shrink=(1,), sigmas=(0.0,), convergence_threshold=-1.0,
                     weights=(0.5, 0.5), metrics=["cc", "mattes"], mi_bins=16)
    warp, inv, recs, _ = O.syn_run(r, g, [f, 1.0 - f], g, [m, 1.0 - m])
    # the energy is the first channel's (CC) value; the weighted energy mixes in the MI value
    assert recs[0].energy != recs[0].energy_weighted
    assert np.isfinite(warp).all()


# ---- preprocess.rs:235-323 (intensity preprocessing) -----------------------------------------

def values_ramp(n):
    return np.arange(n, dtype=np.float64)


def test_preprocess_without_winsorizing_maps_min_to_zero_and_max_just_below_one():
    out = O.preprocess(values_ramp(1000), 0.0, 1.0, 0.0, 1.0)
    assert out[0] == 0.0
    assert abs(out[999] - 999.0 / (999.0 + 999.0 / 2560.0)) < 1e-6
    assert np.all(np.diff(out) > 0)


def test_preprocess_winsorizing_clamps_the_tails_and_is_affine_inside():
    v = values_ramp(1000)
    v[3], v[997] = -5000.0, 9000.0
    out = O.preprocess(v, 0.005, 0.995, 0.0, 1.0)
    assert out[3] == 0.0 and out[997] == 1.0
    lo, hi = O.quantile_window(v, 0.005, 0.995)
    assert -5000.0 < lo < 100.0 and 500.0 < hi < 9000.0
    assert abs(out[500] - (500.0 - lo) / (hi - lo)) < 1e-12


def test_quantile_interpolates_inside_the_bin_like_itk():
    lo, hi = O.quantile_window(values_ramp(2560), 0.25, 0.75)
    assert abs(lo - 640.0) < 5.0 and abs(hi - 1920.0) < 5.0


def test_preprocess_output_range_and_degenerate_inputs():
    out = O.preprocess(values_ramp(100), 0.0, 1.0, -1.0, 3.0)
    assert out[0] == -1.0 and 2.99 < out[99] < 3.0
    for bad in (np.full(10, 2.0), np.zeros(0), np.array([np.nan, np.inf])):
        with pytest.raises(O.OracleError):
            O.preprocess(bad, 0.0, 1.0, 0.0, 1.0)
    mixed = O.preprocess(np.array([1.0, 3.0, np.nan]), 0.0, 1.0, 0.0, 1.0)
    assert mixed[0] == 0.0 and 0.99 < mixed[1] < 1.0 and np.isnan(mixed[2])


def test_preprocess_is_invariant_to_affine_intensity_changes():
    v = ((np.arange(500) * 37) % 101).astype(np.float64)
    a = O.preprocess(v, 0.005, 0.995)
    b = O.preprocess(3.0 * v + 40.0, 0.005, 0.995)
    assert np.abs(a - b).max() < 1e-5


def test_the_unwinsorized_window_reaches_past_the_maximum():
    v = np.append(np.arange(101, dtype=np.float64), 9000.0)
    lo, hi = O.quantile_window(v, 0.0, 1.0)
    assert lo == 0.0 and hi > 9000.0
    assert O.preprocess(v, 0.005, 0.995)[101] == 1.0
    assert O.preprocess(v, 0.0, 1.0)[101] < 1.0


def _window_by_loops(values, lower, upper):
    """Small-case restatement of preprocess.rs:46-173 in plain Python loops (float32 steps in
    numpy float32), the independent check of the oracle's histogram and quantile walk."""
    f32 = np.float32
    fin = [float(x) for x in values if math.isfinite(x)]
    lo, hi = min(fin), max(fin)
    upper_edge = hi + ((hi - lo) / 256.0) / 10.0
    interval = f32(f32(f32(upper_edge) - f32(lo)) / f32(256.0))
    mn = [lo + float(f32(f32(j) * interval)) for j in range(256)]
    mx = [lo + float(f32(f32(j + 1) * interval)) for j in range(255)] + [upper_edge]
    freq = [0.0] * 256
    for x in fin:
        if x < mn[0]:
            b = 0
        elif x >= mx[255]:
            b = 255
        else:
            b = max(sum(1 for m in mn if m <= x) - 1, 0)
        freq[b] += 1.0
    total = sum(freq)

    def quantile(p):
        cum, p_prev = 0.0, 0.0
        if p < 0.5:
            n, p_n = 0, 0.0
            while True:
                f_n = freq[n]
                cum += f_n
                p_prev, p_n = p_n, cum / total
                n += 1
                if not (n < 256 and p_n < p):
                    break
            return mn[n - 1] + ((p - p_prev) / (f_n / total)) * (mx[n - 1] - mn[n - 1])
        n, m, p_n = 255, 0, 1.0
        while True:
            f_n = freq[n]
            cum += f_n
            p_prev, p_n = p_n, 1.0 - cum / total
            n -= 1
            m += 1
            if not (m < 256 and p_n > p):
                break
        b = n + 1
        return mx[b] - ((p_prev - p) / (f_n / total)) * (mx[b] - mn[b])

    return (float(f32(quantile(float(f32(lower))))), float(f32(quantile(float(f32(upper))))))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_the_quantile_window_matches_a_loop_restatement_bit_for_bit(seed):
    rng = np.random.default_rng(seed)
    v = rng.gamma(2.0, 50.0, 3000).astype(np.float32).astype(np.float64)
    v[rng.integers(0, 3000, 20)] = np.nan
    for lower, upper in ((0.0, 1.0), (0.005, 0.995), (0.25, 0.75), (0.6, 0.9)):
        assert O.quantile_window(v, lower, upper) == _window_by_loops(v, lower, upper)


# ---- register.rs:432-470 (isotropic resampling) ----------------------------------------------

def iso_blob_volume(n, spacing, shift):
    """register.rs:432-445: a Gaussian blob plus a hashed noise term."""
    g = O.make_grid((n, n, n), (spacing,) * 3)
    c = (n - 1) * spacing / 2.0
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    lin = (i + n * (j + n * k)).astype(np.uint64)
    r2 = (i * spacing - c - shift) ** 2 + (j * spacing - c) ** 2 + (k * spacing - c) ** 2
    noise = ((lin * np.uint64(2654435761)) % np.uint64(1000)).astype(np.float64) / 20000.0
    return g, np.exp(-r2 / (2.0 * (0.25 * n * spacing) ** 2)) + noise


def test_isotropic_resample_follows_the_pipeline_grid_rule():
    g, v = iso_blob_volume(21, 0.5, 0.0)
    rg, r = O.resample_isotropic(g, v, 1.0)
    assert tuple(rg.size) == (11, 11, 11) and tuple(rg.spacing) == (1.0, 1.0, 1.0)
    assert tuple(rg.origin) == tuple(g.origin)
    assert abs(r[5, 4, 3] - v[10, 8, 6]) < 1e-6
    sg, same = O.resample_isotropic(rg, r, 1.0)
    assert tuple(sg.size) == tuple(rg.size) and np.array_equal(same, r)


def test_isotropic_resample_interpolates_between_source_voxels():
    g = O.make_grid((4, 1, 1), (1.5, 1.0, 1.0))
    rg, r = O.resample_isotropic(g, np.array([0.0, 3.0, 6.0, 9.0]).reshape(1, 1, 4), 1.0)
    assert tuple(rg.size) == (5, 1, 1)
    assert np.abs(r.ravel() - [0.0, 2.0, 4.0, 6.0, 8.0]).max() < 1e-6


def test_isotropic_resample_rejects_a_non_positive_spacing():
    g, v = iso_blob_volume(5, 2.0, 0.0)
    for mm in (0.0, -1.0, math.nan):
        with pytest.raises(O.OracleError):
            O.resample_isotropic(g, v, mm)


# ---- run_syn_from: a later SyN stage through the earlier stages' field (syn.rs:620-660, 761-986)

def test_a_zero_prior_leaves_the_syn_run_unchanged_and_a_real_prior_starts_closer():
    n = 20
    g = cube(n)
    f, m, _ = _cavity_pair(n)
    r = O.syn_recipe(gradient_step=0.25, update_variance=3.0, cc_radius=2, iterations=(4, 3),
                     shrink=(2, 1), sigmas=(1.0, 0.0), convergence_threshold=-1.0)
    w0, i0, r0, last = O.syn_run(r, g, [f], g, [m])
    zero = np.zeros(O.grid_shape(last) + (3,))
    w1, i1, r1, _ = O.syn_run(r, g, [f], g, [m], prior=(last, zero, zero))
    assert np.abs(w1 - w0).max() < 1e-9 and np.abs(i1 - i0).max() < 1e-9
    assert max(abs(a.energy - b.energy) for a, b in zip(r0, r1)) < 1e-12
    # the second stage from the first one's fields: it starts better aligned, and its result is
    # the collapse of its own fields with the prior
    w2, i2, r2, _ = O.syn_run(r, g, [f], g, [m], prior=(last, w0, i0))
    assert r2[0].energy < r0[0].energy
    assert np.abs(w2 - w0).max() > 1e-3
    with pytest.raises(O.OracleError, match="not on the grid of this stage's last level"):
        coarse = O.syn_level_grid(r, g, 0)
        z = np.zeros(O.grid_shape(coarse) + (3,))
        O.syn_run(r, g, [f], g, [m], prior=(coarse, z, z))
