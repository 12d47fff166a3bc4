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


def test_sampled_mi_at_the_config2_finest_level_matches_the_oracle(backend):
    """Config 2's finest level at full size: 25 % regular sampling of the 193 x 229 x 193 head
    phantom, 32 bins -- about 2.13 M samples, so the 2^-32 fixed-point histograms are merged
    from hundreds of blocks and the twelve gradient moments reduce over the full cloud. Against
    the oracle on the same samples: value 1e-5 and derivative 5e-4 relative, valid-sample counts
    exact, for the phantom's own affine map and an Euler transform. The level the product
    prepares itself from device images (fw_mi_level_prepare_regular: sampling, binning and
    fixed bins on the device) holds the oracle's prepared set -- the same 2.13 M points in the
    same order, every fixed bin and the binning equal -- and evaluates the same value on the same
    number of samples."""
    from fastwarp_b200.phantoms import head_pair
    g, fixed, mg, moving, initial = head_pair()
    og = O.make_grid(tuple(g.size), tuple(g.spacing), tuple(g.origin))
    omg = O.make_grid(tuple(mg.size), tuple(mg.spacing), tuple(mg.origin),
                      np.array(mg.direction[:]).reshape(3, 3))
    f64, m64 = fixed.astype(np.float64), moving.astype(np.float64)
    pts = O.sample_points_regular(og, 0.25, 1)
    kept, fbin, b = O.prepare_samples(og, f64, omg, m64, pts, 32)
    assert len(fbin) > 2_000_000
    level = CudaLinearEngine(backend).prepare_level(mg, m64, kept, fbin, b)
    center = tuple(g.origin[a] + 0.5 * (g.size[a] - 1) * g.spacing[a] for a in range(3))
    M = np.array(initial.matrix[:]).reshape(3, 3)
    t_vec = np.array(initial.offset[:]) - np.array(center) + M @ np.array(center)
    cases = [dict(kind="affine", parameters=list(M.ravel()) + list(t_vec), center=center),
             dict(kind="euler", parameters=[0.03, -0.05, 0.02, 2.0, -3.0, 1.5], center=center)]
    for kw in cases:
        v, d = level.value_and_derivative(linear_transform(**kw))
        wv, wd, wn, _ = O.mi_evaluate(b, omg, m64, kept, fbin, O.linear_transform(**kw))
        print(f"{kw['kind']}: value {v:.10f} (oracle {wv:.10f}), |dv| {abs(v - wv):.2e}, "
              f"rel gradient {np.linalg.norm(d - wd) / np.linalg.norm(wd):.2e}, valid {wn}")
        assert abs(v - wv) <= 1e-5 * abs(wv)
        assert np.linalg.norm(d - wd) <= 5e-4 * np.linalg.norm(wd)
        assert level.num_valid() == wn
    fi, mi = backend.upload_image(g, fixed), backend.upload_image(mg, moving)
    own = CudaLinearEngine(backend).prepare_level_regular(g, fi, mi, 0.25, 1, 32)
    dpts, dfb, db = own.samples()
    assert len(dfb) == len(fbin)
    assert np.array_equal(dfb, fbin)
    assert np.abs(dpts - kept).max() < 1e-4  # float32 offsets from the cloud centre
    for k in ("fixed_min", "fixed_max", "moving_min", "moving_max", "fixed_bin_size",
              "moving_bin_size", "fixed_normalized_min", "moving_normalized_min"):
        assert getattr(db, k) == getattr(b, k), k
    t0 = linear_transform(**cases[0])
    assert abs(own.value(t0) - level.value(t0)) <= 1e-12 * abs(level.value(t0))
    assert own.num_valid() == level.num_valid()


def test_all_samples_outside_is_an_error(backend):
    from fastwarp_b200 import FastwarpError
    og, g, f, m, kept, fbin, b = setup()
    level = CudaLinearEngine(backend).prepare_level(g, m, kept, fbin, b)
    far = linear_transform("euler", [0, 0, 0, 500.0, 0, 0])
    with pytest.raises(FastwarpError, match="all samples map outside"):
        level.value(far)


# ---- dense Mattes MI pair of the SyN stage (Backend::mi_value_derivative_pair[_masked]) -------
# cpu/mod.rs:352-381: evaluate_dense twice, (fixed, moving) then (moving, fixed), identity
# transforms, masks on the images' grid. Oracle: the f64 dense restatement pinned against the
# reference's ITK fixtures (tests/test_oracle.py::test_dense_mattes_matches_itk). Tolerances:
# value 1e-5 relative, derivative 5e-4 of its largest component (parity.rs:45-48).

def dense_case(size=(21, 19, 17), spacing=(1.2, 1.0, 1.4), direction=None, seed=5):
    og = O.make_grid(size, spacing, (-4.0, 3.0, 1.5), direction)
    g = make_grid(size, spacing, (-4.0, 3.0, 1.5), direction)
    rng = np.random.default_rng(seed)
    nx, ny, nz = size
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    f = 2.0 + np.sin(0.33 * x) * np.cos(0.27 * y) + 0.7 * np.sin(0.21 * z + 0.1 * x)
    m = 2.0 + np.sin(0.33 * (x - 0.6) + 0.1) * np.cos(0.27 * (y + 0.5)) + \
        0.7 * np.sin(0.21 * (z - 0.3) + 0.1 * x) + 0.02 * rng.standard_normal(f.shape)
    return og, g, f.astype(np.float32), m.astype(np.float32)


def oracle_pair(og, f, m, bins, fm=None, mm=None):
    zero = np.zeros(f.shape + (3,))
    f64, m64 = f.astype(np.float64), m.astype(np.float64)
    a = O.mi_dense(og, f64, og, m64, zero, bins, og if fm is not None else None, fm,
                   og if mm is not None else None, mm)
    b = O.mi_dense(og, m64, og, f64, zero, bins, og if mm is not None else None, mm,
                   og if fm is not None else None, fm)
    return a, b


@pytest.mark.parametrize("bins", [32, 12])
@pytest.mark.parametrize("oblique", [False, True])
def test_dense_mi_pair_matches_the_oracle(backend, bins, oblique):
    og, g, f, m = dense_case(direction=rot_z(0.2) @ rot_x(-0.1) if oblique else None)
    fi, mi = backend.upload_image(g, f), backend.upload_image(g, m)
    ((v0, d0), (v1, d1)), norms = backend.mi_value_derivative_pair_with_norms(fi, mi, bins)
    (w0, n0, e0), (w1, n1, e1) = oracle_pair(og, f, m, bins)
    assert abs(v0 - w0) <= 1e-5 * abs(w0) and abs(v1 - w1) <= 1e-5 * abs(w1)
    g0, g1 = backend.download_field(d0), backend.download_field(d1)
    assert np.abs(g0 - e0).max() <= 5e-4 * np.abs(e0).max()
    assert np.abs(g1 - e1).max() <= 5e-4 * np.abs(e1).max()
    assert abs(norms[0] - np.sqrt((e0 ** 2).sum())) <= 5e-4 * np.sqrt((e0 ** 2).sum())
    (u0, c0), (u1, c1) = backend.mi_value_derivative_pair(fi, mi, bins)
    assert (u0, u1) == (v0, v1)
    assert np.array_equal(backend.download_field(c0), g0)


def test_masked_dense_mi_pair_matches_the_oracle(backend):
    og, g, f, m = dense_case(seed=9)
    nz, ny, nx = f.shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    fm = ((x - 8) ** 2 + (y - 9) ** 2 + (z - 8) ** 2 > 16).astype(np.float64)
    mm = (x < nx - 3).astype(np.float64) * 2.0  # any non-zero value is inside
    fi, mi = backend.upload_image(g, f), backend.upload_image(g, m)
    fmi, mmi = backend.upload_image(g, fm), backend.upload_image(g, mm)
    (v0, d0), (v1, d1) = backend.mi_value_derivative_pair_masked(fi, mi, fmi, mmi, 32)
    (w0, n0, e0), (w1, n1, e1) = oracle_pair(og, f, m, 32, fm, mm)
    assert abs(v0 - w0) <= 1e-5 * abs(w0) and abs(v1 - w1) <= 1e-5 * abs(w1)
    g0, g1 = backend.download_field(d0), backend.download_field(d1)
    assert np.abs(g0 - e0).max() <= 5e-4 * np.abs(e0).max()
    assert np.abs(g1 - e1).max() <= 5e-4 * np.abs(e1).max()
    outside = (fm == 0) | (mm == 0)
    assert np.all(g0[outside] == 0.0) and np.all(g1[outside] == 0.0)
    # masks of ones are no masks
    ones = backend.upload_image(g, np.ones(f.shape, np.float32))
    (a0, b0), (a1, b1) = backend.mi_value_derivative_pair_masked(fi, mi, ones, ones, 32)
    (p0, q0), (p1, q1) = backend.mi_value_derivative_pair(fi, mi, 32)
    assert (a0, a1) == (p0, p1)
    assert np.array_equal(backend.download_field(b0), backend.download_field(q0))


def test_dense_mi_errors_carry_the_reference_messages(backend):
    from fastwarp_b200 import FastwarpError
    og, g, f, m = dense_case(size=(9, 8, 7))
    fi, mi = backend.upload_image(g, f), backend.upload_image(g, m)
    const = backend.upload_image(g, np.full(f.shape, 3.0, np.float32))
    with pytest.raises(FastwarpError, match="the fixed image is constant"):
        backend.mi_value_derivative_pair(const, mi, 32)
    with pytest.raises(FastwarpError, match="the moving image is constant"):
        backend.mi_value_derivative_pair(fi, const, 32)
    with pytest.raises(FastwarpError, match="at least five histogram bins"):
        backend.mi_value_derivative_pair(fi, mi, 4)
    zeros = backend.upload_image(g, np.zeros(f.shape, np.float32))
    with pytest.raises(FastwarpError, match="no finite fixed-image voxel lies inside the fixed mask"):
        backend.mi_value_derivative_pair_masked(fi, mi, zeros, None, 32)
    half = np.zeros(f.shape, np.float32)
    half[:, :, :4] = 1.0
    other = 1.0 - half
    with pytest.raises(FastwarpError, match="no voxel of the registration level lies inside"):
        backend.mi_value_derivative_pair_masked(fi, mi, backend.upload_image(g, half),
                                                backend.upload_image(g, other), 32)


# ---- the linear-stage optimiser on the device MI level (optimizer.rs:311-435) ---------------
def test_level_optimiser_matches_the_callback_path_and_follows_the_oracle(backend):
    """fw_mi_level_optimize against (a) the same optimiser driven through Python callbacks over
    the same device level (bit-identical: the evaluations are deterministic) and (b) the oracle's
    optimiser over the f64 oracle MI: the MI values agree to 1e-5 relative, so the trajectories
    stay together over a short level; the final transforms agree to 0.02 mm at the corners."""
    from fastwarp_b200.backend import cg_settings_ants, grid_corners, mi_level_optimize, \
        optimize_level
    og, g, f, m, kept, fbin, b = setup(size=(32, 30, 28), spacing=(1.0, 1.0, 1.0),
                                       origin=(0, 0, 0), direction=np.eye(3), seed=5)
    level = CudaLinearEngine(backend).prepare_level(g, m, kept, fbin, b)
    center = (15.5, 14.5, 13.5)
    start = [0.02, -0.01, 0.015, 0.6, -0.4, 0.3]
    corners = grid_corners(g)
    settings = cg_settings_ants(0.1, 12, -1.0, 10)
    t, trace = mi_level_optimize(level, corners, linear_transform("euler", start, center=center),
                                 settings)
    assert trace["iterations"] == 12 and trace["line_search_evaluations"] > 0
    assert trace["values"][-1] < trace["values"][0]
    t2, trace2 = optimize_level(level.value, level.value_and_derivative, corners,
                                linear_transform("euler", start, center=center), settings)
    assert trace2["values"] == trace["values"]
    assert list(t2.parameters[:6]) == list(t.parameters[:6])

    def ov(tt):
        return O.mi_evaluate(b, og, m, kept, fbin, tt, False)[0]

    def ovd(tt):
        v, d, _, _ = O.mi_evaluate(b, og, m, kept, fbin, tt)
        return v, d
    ot, otrace = O.cg_optimize_level(ov, ovd, corners,
                                     O.linear_transform("euler", start, center=center),
                                     O.cg_settings_ants(0.1, 12, -1.0, 10))
    assert otrace["iterations"] == 12
    assert abs(trace["values"][0] - otrace["values"][0]) <= 1e-5 * abs(otrace["values"][0])
    assert abs(trace["best_value"] - otrace["best_value"]) <= 1e-4 * abs(otrace["best_value"])
    ma, oa = O.linear_map(O.linear_transform("euler", list(t.parameters[:6]), center=center))
    mb, ob = O.linear_map(ot)
    shift = max(np.linalg.norm((ma - mb) @ c + oa - ob) for c in corners)
    assert shift < 0.02, shift
