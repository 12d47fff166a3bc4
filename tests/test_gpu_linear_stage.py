"""One linear stage (run_linear_stage, linear.rs:512-597) and the rigid + affine chain
(run_linear_chain, linear.rs:1105-1212) on the device against the oracle's
pieces composed the same way: per level the shrunk virtual grid, Deriche smoothing, regular
sampling with the stage's seed sequence, sample preparation and the conjugate-gradient optimiser
over Mattes MI.

The device smooths into float32 images and evaluates MI in float32 with f64 reductions, the oracle
in f64, so the bars are those of the level-optimiser test: each level's best MI value to 1e-4
relative, the prepared sample counts to 0.5 %, the final transforms to 0.05 mm at the level grid's
corners.
"""
import numpy as np
import pytest

import oracle as O
from fastwarp_b200 import FastwarpError, linear_transform, make_grid
from fastwarp_b200 import _native as N
from fastwarp_b200.backend import (grid_corners, linear_recipe, run_linear_chain,
                                   run_linear_stage)
from fastwarp_b200.phantoms import blob_pair

pytestmark = pytest.mark.gpu


def ogrid(g):
    return O.make_grid(tuple(g.size), tuple(g.spacing), tuple(g.origin),
                       np.array(g.direction[:]).reshape(3, 3))


def oracle_stage(g, fixed, moving, kind, start, center, iterations, shrink, sigmas, step=0.1,
                 pct=0.25, bins=32, seed=1, outer=(np.eye(3), (0, 0, 0), (0, 0, 0)), mask=None):
    """run_linear_stage restated over the oracle's pieces (sigmas in voxels); `outer` is the
    earlier transforms as (matrix, translation, centre); `mask` (grid, values) keeps only the
    sample points inside it (linear.rs:940-945). A level left without a sample point reports
    samples 0 and no values."""
    og = ogrid(g)
    fixed, moving = fixed.astype(np.float64), moving.astype(np.float64)
    t = O.linear_transform(kind, start, center=center, outer_matrix=outer[0],
                           outer_translation=outer[1], outer_center=outer[2])
    out = []
    for level, (its, sf, sg) in enumerate(zip(iterations, shrink, sigmas)):
        f = O.shrink_factors(sf, tuple(g.spacing))
        lg = O.shrink_grid(og, f)
        if sg > 0:
            s = tuple(sg * x for x in g.spacing)
            fs, ms = O.smooth_recursive(og, fixed, s), O.smooth_recursive(og, moving, s)
        else:
            fs, ms = fixed, moving
        pts = O.sample_points_regular(lg, pct, seed + level)
        if mask is not None:
            pts = pts[O.mask_inside(mask[0], mask[1], pts)]
            if len(pts) == 0:
                out.append(dict(samples=0, values=[], corners=grid_corners(lg)))
                continue
        kept, fbin, b = O.prepare_samples(og, fs, og, ms, pts, bins)

        def ov(tt):
            return O.mi_evaluate(b, og, ms, kept, fbin, tt, False)[0]

        def ovd(tt):
            v, d, _, _ = O.mi_evaluate(b, og, ms, kept, fbin, tt)
            return v, d
        corners = grid_corners(lg)
        t, trace = O.cg_optimize_level(ov, ovd, corners, t,
                                       O.cg_settings_ants(step, its, 1e-6, 10))
        out.append(dict(samples=len(fbin), values=trace["values"], corners=corners))
    return t, out


def corner_shift(t_dev, t_orc, corners):
    ma, oa = O.linear_map(O.linear_transform("euler" if t_dev.kind == 0 else "affine",
                                             list(t_dev.parameters[:6 if t_dev.kind == 0 else 12]),
                                             center=tuple(t_dev.center)))
    mb, ob = O.linear_map(t_orc)
    return max(np.linalg.norm((ma - mb) @ c + oa - ob) for c in corners)


@pytest.mark.parametrize("kind", ["euler", "affine"])
def test_a_linear_stage_matches_the_oracle(backend, kind):
    g, fixed, moving = blob_pair(48, seed=77)
    center = tuple((s - 1) * sp / 2.0 for s, sp in zip(g.size, g.spacing))
    start = [0.0] * 6 if kind == "euler" else list(np.eye(3).ravel()) + [0.0] * 3
    its, shrink, sigmas = (12, 8), (2, 1), (1.0, 0.0)
    r = linear_recipe(iterations=its, shrink_factors=shrink, smoothing_sigmas=sigmas)
    t, levels = run_linear_stage(backend, r, backend.upload_image(g, fixed),
                                 backend.upload_image(g, moving),
                                 linear_transform(kind, start, center=center))
    ot, olevels = oracle_stage(g, fixed, moving, kind, start, center, its, shrink, sigmas)
    assert [lv["skipped"] for lv in levels] == [False, False]
    for lv, ol in zip(levels, olevels):
        assert abs(lv["samples"] - ol["samples"]) <= 0.005 * ol["samples"]
        best = min(ol["values"])
        assert abs(lv["best_value"] - best) <= 1e-4 * abs(best), (lv["best_value"], best)
    assert levels[0]["iterations"] > 0 and levels[1]["iterations"] > 0
    shift = corner_shift(t, ot, olevels[-1]["corners"])
    print(f"{kind}: corner shift {shift:.2e} mm, best MI {levels[-1]['best_value']:.6f} "
          f"(oracle {min(olevels[-1]['values']):.6f}), samples {levels[-1]['samples']}")
    assert shift < 0.05, shift
    # the stage moved the transform
    assert max(abs(p - s) for p, s in zip(levels[-1]["parameters"], start)) > 1e-4


def test_a_stage_whose_levels_all_see_one_fixed_value_is_refused(backend):
    g, _, moving = blob_pair(24, seed=3)
    flat = np.full(tuple(g.size)[::-1], 0.5, np.float32)
    r = linear_recipe(iterations=(5,), shrink_factors=(1,), smoothing_sigmas=(0.0,))
    with pytest.raises(FastwarpError, match="every level of the rigid stage has too few usable"):
        run_linear_stage(backend, r, backend.upload_image(g, flat),
                         backend.upload_image(g, moving),
                         linear_transform("euler", [0.0] * 6, center=(11.5, 11.5, 11.5)))


def inner_map(t):
    """The optimised part of a stage's transform alone, as (matrix, offset)."""
    n = 6 if t.kind == 0 else 12
    return O.linear_map(O.linear_transform("euler" if t.kind == 0 else "affine",
                                           list(t.parameters[:n]), center=tuple(t.center)))


def test_the_linear_chain_composes_its_stages_and_follows_the_oracle(backend):
    """run_linear_chain (linear.rs:1148-1212): the centre-of-mass start, the rigid stage, the
    affine stage from the rigid result, the collapsed total. Checked exactly: each of the chain's
    stages is run_linear_stage from the chain's own start transform, bit for bit (the affine stage
    takes the rigid stage's smoothed moving images and samples from the chain's cache, which equal
    a fresh preparation); the initial transform is the centres of mass (1e-9 mm against numpy);
    the total is the collapse of the three (1e-9 mm at the grid corners against the same
    composition in numpy). Against the oracle's chain the total stays within 0.5 mm at the
    corners: each stage alone is held to 0.05 mm by the stage tests, but two conjugate-gradient
    runs of 10 + 6 iterations whose line searches compare MI values that agree to ~1e-7 can
    branch differently at a near-tie, and the second stage starts from the first one's result."""
    g, fixed, moving = blob_pair(40, seed=29)
    its, shrink, sigmas = (10, 6), (2, 1), (1.0, 0.0)
    r = linear_recipe(iterations=its, shrink_factors=shrink, smoothing_sigmas=sigmas)
    fi, mi = backend.upload_image(g, fixed), backend.upload_image(g, moving)
    out = run_linear_chain(backend, r, r, fi, mi, fi, mi)
    assert out["affine_samples_cached"] == [True, True]
    nz, ny, nx = fixed.shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    pts = [g.origin[a] + g.spacing[a] * v for a, v in enumerate((x, y, z))]

    def cog(v):
        v = v.astype(np.float64)
        return np.array([(p * v).sum() for p in pts]) / v.sum()
    fc, mc = cog(fixed), cog(moving)
    assert np.abs(out["initial"][2] - fc).max() < 1e-9
    assert np.abs(out["initial"][1] - (mc - fc)).max() < 1e-9
    # each stage is the stage run alone from the chain's start transform
    for key, n, start in (("rigid", 6, [0.0] * 6), ("affine", 12, list(np.eye(3).ravel()) + [0.0] * 3)):
        t0 = N.LinearTransform.from_buffer_copy(out[key + "_transform"])
        for k in range(12):
            t0.parameters[k] = start[k] if k < n else 0.0
        alone, _ = run_linear_stage(backend, r, fi, mi, t0)
        assert list(alone.parameters[:n]) == out[key], key
    # the collapse of the three
    corners = grid_corners(g)
    mr, offr = inner_map(out["rigid_transform"])
    off_after = offr + out["initial"][1]
    ma, offa = inner_map(out["affine_transform"])
    total_m, total_off = mr @ ma, mr @ offa + off_after
    dm, dt, dc = out["total"]
    collapse = max(np.linalg.norm((dm @ (c - dc) + dc + dt) - (total_m @ c + total_off))
                   for c in corners)
    assert collapse < 1e-9, collapse
    assert np.abs(dc - out["initial"][2]).max() == 0.0  # the total keeps the affine stage's centre
    assert max(abs(v) for v in out["rigid"]) > 1e-4  # the rigid stage moved
    # the oracle's chain
    rt, _ = oracle_stage(g, fixed, moving, "euler", [0.0] * 6, tuple(fc), its, shrink, sigmas,
                         outer=(np.eye(3), tuple(mc - fc), tuple(fc)))
    omr, ooffr = inner_map(rt)
    ooff_after = ooffr + (mc - fc)
    at, _ = oracle_stage(g, fixed, moving, "affine", list(np.eye(3).ravel()) + [0.0] * 3,
                         tuple(fc), its, shrink, sigmas, outer=(omr, tuple(ooff_after), (0, 0, 0)))
    oma, ooffa = inner_map(at)
    om, ooff = omr @ oma, omr @ ooffa + ooff_after
    shift = max(np.linalg.norm((dm @ (c - dc) + dc + dt) - (om @ c + ooff)) for c in corners)
    print(f"chain: corner shift against the oracle's chain {shift:.2e} mm")
    assert shift < 0.5, shift


def half_mask(g):
    """linear.rs:1546-1576: the voxels of the upper half along x."""
    nx, ny, nz = g.size
    m = np.zeros((nz, ny, nx), np.float32)
    m[:, :, nx // 2:] = 1.0
    return m


@pytest.mark.parametrize("kind", ["euler", "affine"])
def test_a_masked_linear_stage_matches_the_oracle(backend, kind):
    """The fixed mask (LinearRecipe::mask): only the jittered sample points whose nearest mask
    voxel is inside are kept (linear.rs:940-945); the sample set shrinks (linear.rs:1546-1576)
    and the stage follows the oracle's on the kept points. The mask has its own grid, coarser
    and shifted against the fixed image's, as ANTs attaches it in physical space."""
    g, fixed, moving = blob_pair(48, seed=77)
    mg = make_grid((24, 24, 24), spacing=tuple(2.0 * s for s in g.spacing),
                   origin=tuple(o + 0.3 for o in g.origin))
    mask = half_mask(mg)
    mask[:, :4, :] = 0.0  # and a slab off the bottom rows
    center = tuple((s - 1) * sp / 2.0 for s, sp in zip(g.size, g.spacing))
    start = [0.0] * 6 if kind == "euler" else list(np.eye(3).ravel()) + [0.0] * 3
    its, shrink, sigmas = (12, 8), (2, 1), (1.0, 0.0)
    r = linear_recipe(iterations=its, shrink_factors=shrink, smoothing_sigmas=sigmas)
    fi, mi = backend.upload_image(g, fixed), backend.upload_image(g, moving)
    _, base = run_linear_stage(backend, r, fi, mi, linear_transform(kind, start, center=center))
    t, levels = run_linear_stage(backend, r, fi, mi, linear_transform(kind, start, center=center),
                                 fixed_mask=backend.upload_image(mg, mask))
    omg = ogrid(mg)
    ot, olevels = oracle_stage(g, fixed, moving, kind, start, center, its, shrink, sigmas,
                               mask=(omg, mask))
    for lv, bl, ol in zip(levels, base, olevels):
        assert 0 < lv["samples"] < 0.6 * bl["samples"]
        assert abs(lv["samples"] - ol["samples"]) <= 0.005 * ol["samples"]
        best = min(ol["values"])
        assert abs(lv["best_value"] - best) <= 1e-4 * abs(best), (lv["best_value"], best)
    shift = corner_shift(t, ot, olevels[-1]["corners"])
    print(f"masked {kind}: corner shift {shift:.2e} mm, samples {[lv['samples'] for lv in levels]}"
          f" of {[b['samples'] for b in base]}")
    assert shift < 0.05, shift


def plane_mask_missed_by_coarse_level(g, shrink, seed=1):
    """After linear.rs:1578-1596: a one-voxel plane x = const of the fixed grid that none of the
    coarse level's jittered sample points (the stage's first seed) rounds to."""
    og = ogrid(g)
    pts = O.sample_points_regular(O.shrink_grid(og, O.shrink_factors(shrink, tuple(g.spacing))),
                                  0.25, seed)
    hit = {int(np.floor(O.point_to_index(og, p)[0] + 0.5)) for p in pts}
    plane = next(x for x in range(2, g.size[0] - 2) if x not in hit)
    m = np.zeros(tuple(g.size)[::-1], np.float32)
    m[:, :, plane] = 1.0
    return m


def test_a_level_without_masked_samples_is_skipped_and_a_stage_of_only_such_levels_fails(backend):
    """linear.rs:1598-1640: the coarse level keeps no sample point inside a thin plane mask and is
    skipped (samples 0, no iteration, the start unchanged); the fine level runs. A stage whose
    only level is skipped fails with the reference's reason."""
    g, fixed, moving = blob_pair(30, seed=5)
    mask = plane_mask_missed_by_coarse_level(g, 6)
    fi, mi = backend.upload_image(g, fixed), backend.upload_image(g, moving)
    m = backend.upload_image(g, mask)
    start = linear_transform("euler", [0.0] * 6, center=(14.5, 14.5, 14.5))
    r = linear_recipe(iterations=(5, 5), shrink_factors=(6, 1), smoothing_sigmas=(0.0, 0.0))
    t, levels = run_linear_stage(backend, r, fi, mi, start, fixed_mask=m)
    opts = O.sample_points_regular(O.shrink_grid(ogrid(g), O.shrink_factors(6, (1.0,) * 3)),
                                   0.25, 1)
    assert not O.mask_inside(ogrid(g), mask, opts).any()
    assert levels[0]["skipped"] and levels[0]["samples"] == 0 and levels[0]["iterations"] == 0
    assert levels[0]["parameters"] == [0.0] * 6
    assert not levels[1]["skipped"] and levels[1]["samples"] > 0
    coarse = linear_recipe(iterations=(5,), shrink_factors=(6,), smoothing_sigmas=(0.0,))
    with pytest.raises(FastwarpError, match="no sample point lands on the fixed image inside the "
                                            "fixed mask"):
        run_linear_stage(backend, coarse, fi, mi, start, fixed_mask=m)
    with pytest.raises(FastwarpError, match="fixed mask has no voxel inside"):
        run_linear_stage(backend, coarse, fi, mi, start,
                         fixed_mask=backend.upload_image(g, np.zeros_like(mask)))


def test_the_masked_linear_chain_keeps_its_samples_inside_the_mask(backend):
    """The chain passes the fixed mask to both stages."""
    g, fixed, moving = blob_pair(40, seed=29)
    r = linear_recipe(iterations=(6, 4), shrink_factors=(2, 1), smoothing_sigmas=(1.0, 0.0))
    fi, mi = backend.upload_image(g, fixed), backend.upload_image(g, moving)
    m = backend.upload_image(g, half_mask(g))
    full = run_linear_chain(backend, r, r, fi, mi, fi, mi)
    masked = run_linear_chain(backend, r, r, fi, mi, fi, mi, fixed_mask=m)
    for key in ("rigid_samples", "affine_samples"):
        for a, b in zip(masked[key], full[key]):
            assert 0 < a < 0.6 * b


@pytest.mark.parametrize("masked", [False, True])
def test_the_device_sample_preparation_matches_the_oracle(backend, masked):
    """fw_mi_level_prepare_regular draws the regular sample set and prepares it on the device
    (the jittered points, the fixed mask, the fixed range at the nearest voxels, the moving range
    over the whole image, the trilinear fixed bins). Against the oracle's sampling and
    preparation of the same float32 images on an oblique, anisotropic grid with a shrunk level
    grid: the binning is equal to the last bit, the same points are kept in the same raster
    order, each within the float32 rounding of its offset from the cloud centre, and every fixed
    bin is equal. (The device's log and cos may differ from the host library's in the last bit;
    that moves a point by ~1e-15 mm, and no point of this set lies that close to an edge.)"""
    from fastwarp_b200.backend import CudaLinearEngine
    rot = np.array([[0.98, -0.17, 0.1], [0.17, 0.985, 0.0], [-0.1, 0.02, 0.995]])
    q, _ = np.linalg.qr(rot)
    g = make_grid((44, 40, 36), (1.1, 0.9, 1.3), (-20.0, 7.5, -11.0), q)
    _, fixed, moving = blob_pair(44, seed=303)
    fixed, moving = fixed[:36, :40, :44].copy(), moving[:36, :40, :44].copy()
    og = ogrid(g)
    lg = O.shrink_grid(og, (2, 2, 1))
    dlg = make_grid(tuple(lg.size), tuple(lg.spacing), tuple(lg.origin),
                    np.array(lg.direction[:]).reshape(3, 3))
    fi, mi = backend.upload_image(g, fixed), backend.upload_image(g, moving)
    mask_img = None
    pts = O.sample_points_regular(lg, 0.25, 7)
    if masked:
        mg = make_grid((20, 22, 18), (2.2, 1.9, 2.5), (-18.0, 8.0, -10.0), q)
        mk = np.zeros((18, 22, 20), np.float32)
        mk[2:15, 3:20, 4:17] = 1.0
        mask_img = backend.upload_image(mg, mk)
        pts = pts[O.mask_inside(ogrid(mg), mk, pts)]
    kept, fbin, ob = O.prepare_samples(og, fixed, og, moving, pts, 32)
    lvl = CudaLinearEngine(backend).prepare_level_regular(dlg, fi, mi, 0.25, 7, 32, mask_img)
    dpts, dfb, db = lvl.samples()
    for k in ("fixed_min", "fixed_max", "moving_min", "moving_max", "fixed_bin_size",
              "moving_bin_size", "fixed_normalized_min", "moving_normalized_min"):
        assert getattr(db, k) == getattr(ob, k), k
    assert len(dfb) == len(fbin) > 1000
    err = np.abs(dpts - kept).max()
    print(f"samples {len(fbin)} of {len(pts)} candidates; largest point difference {err:.2e} mm")
    assert err < 1e-5
    assert np.array_equal(dfb, fbin)
    lvl.free()
