"""Op-by-op parity of the CUDA engine against the f64 oracle, through the C ABI.

Mirrors the reference's GPU parity harness (crates/fastwarp-gpu/src/parity.rs): seeded smooth
content on odd, anisotropic and oblique grids, and its per-op tolerances (parity.rs:25-54),
stated here as the largest absolute error over the reference's range unless noted:
warp 1e-5, CC value 1e-5 relative, CC derivative 1e-4, smoothing 2e-6, norms 1e-6 relative,
scale/axpy 1e-6, compose 1e-5, inversion 1e-4 of the field's range, resample 1e-5.
"""
import numpy as np
import pytest

import oracle as O
from cases import (CASES, continuous_index, edge_distance, field, grid_of, image,
                   vector_at, voxel_points)
from fastwarp_b200 import _native as N
from fastwarp_b200.backend import make_affine, make_grid

pytestmark = pytest.mark.gpu

NAMES = list(CASES)


def fgrid(case):
    return make_grid(case["size"], case["spacing"], case["origin"], case["direction"])


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def worst(a, b):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max())


def assert_only_edge_flips(diff, edge, tol):
    """Every voxel off by more than `tol` samples within one voxel of a buffer face (where the
    f32 field and the two engines' index arithmetic can put a point on either side of ITK's
    inside test); they are rare; every other voxel meets `tol`."""
    bad = diff > tol
    assert np.mean(bad) < 2e-3, np.mean(bad)
    assert edge[bad].max(initial=0.0) < 1.0, edge[bad].max()
    assert diff[edge >= 1.0].max(initial=0.0) <= tol, diff[edge >= 1.0].max()


@pytest.mark.parametrize("name", NAMES)
def test_warp_through_field_matches(backend, name):
    case = CASES[name]
    og, g = grid_of(case), fgrid(case)
    img, fld = image(case), field(case)
    src = backend.upload_image(g, img.astype(np.float32))
    f = backend.upload_field(g, fld)
    out = backend.warp_through_field(src, f).download()
    want = O.warp(og, img, og, fld)
    assert worst(out, want) <= 1e-5 * max(1.0, np.abs(want).max())
    # with an affine after the field
    A = np.array([[0.98, 0.03, 0.0], [-0.02, 1.01, 0.01], [0.0, 0.02, 0.97]])
    off = np.array([0.7, -0.4, 0.3])
    out = backend.warp_through_field(src, f, affine=make_affine(A, off)).download()
    want = O.warp(og, img, og, fld, affine=O.make_affine(A, off))
    diff = np.abs(out - want)
    # the sampled source index of every voxel: c = S^-1 (A (x + u) + off - origin)
    c = continuous_index(case, (voxel_points(case) + fld) @ A.T + off)
    assert_only_edge_flips(diff, edge_distance(case, c), 1e-5 * max(1.0, np.abs(want).max()))


@pytest.mark.parametrize("name", ["selftest", "awkward_oblique"])
def test_warp_with_an_earlier_field_and_masks_matches(backend, name):
    case = CASES[name]
    og, g = grid_of(case), fgrid(case)
    img, fld = image(case), field(case, amp=1.0)
    sz = case["size"]
    pre_case = dict(case, size=(sz[0] - 2, sz[1], sz[2]))
    opg, pg = grid_of(pre_case), fgrid(pre_case)
    pre = field(pre_case, amp=0.8, seed_offset=7)
    src = backend.upload_image(g, img.astype(np.float32))
    f = backend.upload_field(g, fld)
    p = backend.upload_field(pg, pre)
    aff = (np.eye(3) * 1.01, np.array([0.2, -0.1, 0.05]))
    out = backend.warp_through_field(src, f, pre=p, affine=make_affine(*aff)).download()
    want = O.warp(og, img, og, fld, opg, pre, O.make_affine(*aff))
    # two places where a sample can flip: the earlier field's buffer at q = x + u(x), and the
    # source's at c = S^-1 (A (q + pre(q)) + off - origin)
    q = voxel_points(case) + fld
    cq = continuous_index(pre_case, q)
    c = continuous_index(case, (q + vector_at(pre_case, pre, cq)) @ aff[0].T + aff[1])
    near = np.minimum(edge_distance(pre_case, cq), edge_distance(case, c))
    assert_only_edge_flips(np.abs(out - want), near, 1e-5 * max(1.0, np.abs(want).max()))
    mask_img = (img > np.median(img)).astype(np.float64)
    m = backend.upload_image(g, mask_img.astype(np.float32))
    got = backend.warp_mask_through_field(m, f, pre=p, affine=make_affine(*aff)).download()
    want = O.warp_mask(og, mask_img, og, fld, opg, pre, O.make_affine(*aff))
    assert np.mean(got != want) < 2e-3
    prod = backend.upload_image(g, want.astype(np.float32))
    again = backend.warp_mask_through_field(m, f, pre=p, affine=make_affine(*aff), product=prod)
    assert again is prod
    assert np.mean(again.download() != want * want) < 2e-3


@pytest.mark.parametrize("name", NAMES)
def test_cc_pair_matches_in_both_directions(backend, name):
    case = CASES[name]
    og, g = grid_of(case), fgrid(case)
    fimg, mimg = image(case), image(case, seed_offset=5)
    r = case["radius"]
    fi = backend.upload_image(g, fimg.astype(np.float32))
    mi = backend.upload_image(g, mimg.astype(np.float32))
    (v1, d1), (v2, d2) = backend.cc_value_derivative_pair(fi, mi, r)
    (w1, e1), (w2, e2) = O.cc_pair(og, fimg, mimg, r)
    assert rel(v1, w1) <= 1e-5 and rel(v2, w2) <= 1e-5
    g1, g2 = backend.download_field(d1), backend.download_field(d2)
    assert worst(g1, e1) <= 1e-4 * np.abs(e1).max()
    assert worst(g2, e2) <= 1e-4 * np.abs(e2).max()
    # with norms: the same fields and their L2 norms
    ((u1, c1), (u2, c2)), norms = backend.cc_value_derivative_pair_with_norms(fi, mi, r)
    assert (u1, u2) == (v1, v2)
    assert np.array_equal(backend.download_field(c1), g1)
    assert rel(norms[0], np.sqrt((e1 ** 2).sum())) <= 1e-5
    assert rel(norms[1], np.sqrt((e2 ** 2).sum())) <= 1e-5


@pytest.mark.parametrize("name", ["awkward_aligned", "awkward_oblique", "cube_r1"])
@pytest.mark.parametrize("sums", [0, 1])
def test_cc_pair_with_exactly_zero_regions_matches_the_oracle(backend, name, sums):
    """Images that are exactly zero over whole regions (a zero-padded or skull-stripped
    background): the reference sums every window directly (metric/cc.rs:137-157), so a window
    where an image is zero sums to exactly zero and takes the degenerate local CC of 1; the
    engine's running z sums must do the same. Both window-sum arithmetics (float64, compensated
    float32) are checked; the zero regions cover a third of the volume, so a wrong degenerate
    rule moves the value by several per cent."""
    import ctypes as C
    case = CASES[name]
    og, g = grid_of(case), fgrid(case)
    fimg, mimg = image(case), image(case, seed_offset=5)
    nz, ny, nx = fimg.shape
    mimg[:, :, : nx // 3] = 0.0              # the moving image zero on a slab
    fimg[: nz // 4] = 0.0                    # the fixed image zero on another
    mimg[nz // 2:, ny // 2:, nx // 2:] = 0.0  # and both zero in a corner
    fimg[nz // 2:, ny // 2:, nx // 2:] = 0.0
    r = case["radius"]
    fi = backend.upload_image(g, fimg.astype(np.float32))
    mi = backend.upload_image(g, mimg.astype(np.float32))
    N.check(N.lib().fw_set_cc_window_sums(C.c_int32(sums)))
    try:
        (v1, d1), (v2, d2) = backend.cc_value_derivative_pair(fi, mi, r)
    finally:
        N.check(N.lib().fw_set_cc_window_sums(C.c_int32(0)))
    (w1, e1), (w2, e2) = O.cc_pair(og, fimg, mimg, r)
    assert rel(v1, w1) <= 1e-5 and rel(v2, w2) <= 1e-5, (v1, w1)
    assert worst(backend.download_field(d1), e1) <= 1e-4 * np.abs(e1).max()
    assert worst(backend.download_field(d2), e2) <= 1e-4 * np.abs(e2).max()


def test_cc_of_an_image_with_itself_is_minus_one(backend):
    case = CASES["awkward_aligned"]
    g = fgrid(case)
    img = backend.upload_image(g, image(case).astype(np.float32))
    (v, d), _ = backend.cc_value_derivative_pair(img, img, 3)
    assert abs(v + 1.0) < 1e-6
    assert np.abs(backend.download_field(d)).max() < 1e-4


def test_cc_reruns_are_bit_identical(backend):
    case = CASES["awkward_oblique"]
    g = fgrid(case)
    fi = backend.upload_image(g, image(case).astype(np.float32))
    mi = backend.upload_image(g, image(case, seed_offset=5).astype(np.float32))
    (a, da), _ = backend.cc_value_derivative_pair(fi, mi, 4)
    (b, db), _ = backend.cc_value_derivative_pair(fi, mi, 4)
    assert a == b
    assert np.array_equal(backend.download_field(da), backend.download_field(db))


@pytest.mark.parametrize("radius", [1, 5, 6, 8])
def test_cc_every_radius_path_matches(backend, radius):
    case = dict(CASES["awkward_aligned"], radius=radius)
    og, g = grid_of(case), fgrid(case)
    fimg, mimg = image(case), image(case, seed_offset=3)
    fi = backend.upload_image(g, fimg.astype(np.float32))
    mi = backend.upload_image(g, mimg.astype(np.float32))
    (v1, d1), (v2, d2) = backend.cc_value_derivative_pair(fi, mi, radius)
    (w1, e1), (w2, e2) = O.cc_pair(og, fimg, mimg, radius)
    assert rel(v1, w1) <= 1e-5
    assert worst(backend.download_field(d1), e1) <= 1e-4 * np.abs(e1).max()
    assert worst(backend.download_field(d2), e2) <= 1e-4 * np.abs(e2).max()


def ball_mask(case):
    """metric/cc.rs:465-473's mask shape on the case grid: out of a ball, the first x plane and a
    corner strip; the inside value is 3 (any non-zero value counts)."""
    nx, ny, nz = case["size"]
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    d = np.sqrt((i - nx / 2.0) ** 2 + (j - ny / 2.5) ** 2 + (k - nz / 1.8) ** 2)
    out = (d < min(nx, ny, nz) / 3.5) | (i == 0) | ((j == ny - 1) & (k > nz // 2))
    return np.where(out, 0.0, 3.0)


@pytest.mark.parametrize("name", NAMES)
def test_masked_cc_pair_matches(backend, name):
    case = CASES[name]
    og, g = grid_of(case), fgrid(case)
    fimg, mimg = image(case), image(case, seed_offset=5)
    valid = ball_mask(case)
    r = case["radius"]
    fi = backend.upload_image(g, fimg.astype(np.float32))
    mi = backend.upload_image(g, mimg.astype(np.float32))
    vi = backend.upload_image(g, valid.astype(np.float32))
    (v1, d1), (v2, d2) = backend.cc_value_derivative_pair_masked(fi, mi, vi, r)
    (w1, e1), (w2, e2) = O.cc_pair(og, fimg, mimg, r, valid=valid)
    assert rel(v1, w1) <= 1e-5 and rel(v2, w2) <= 1e-5
    g1, g2 = backend.download_field(d1), backend.download_field(d2)
    assert worst(g1, e1) <= 1e-4 * np.abs(e1).max()
    assert worst(g2, e2) <= 1e-4 * np.abs(e2).max()
    assert np.all(g1[valid == 0] == 0.0) and np.all(g2[valid == 0] == 0.0)
    ((u1, c1), (u2, c2)), norms = backend.cc_value_derivative_pair_masked_with_norms(fi, mi, vi, r)
    assert (u1, u2) == (v1, v2)
    assert np.array_equal(backend.download_field(c1), g1)
    assert rel(norms[0], np.sqrt((e1 ** 2).sum())) <= 1e-5
    assert rel(norms[1], np.sqrt((e2 ** 2).sum())) <= 1e-5


@pytest.mark.parametrize("radius", [1, 5, 6, 8])
def test_masked_cc_every_radius_path_matches(backend, radius):
    case = dict(CASES["awkward_aligned"], radius=radius)
    og, g = grid_of(case), fgrid(case)
    fimg, mimg = image(case), image(case, seed_offset=3)
    valid = ball_mask(case)
    fi = backend.upload_image(g, fimg.astype(np.float32))
    mi = backend.upload_image(g, mimg.astype(np.float32))
    vi = backend.upload_image(g, valid.astype(np.float32))
    (v1, d1), (v2, d2) = backend.cc_value_derivative_pair_masked(fi, mi, vi, radius)
    (w1, e1), (w2, e2) = O.cc_pair(og, fimg, mimg, radius, valid=valid)
    assert rel(v1, w1) <= 1e-5
    assert worst(backend.download_field(d1), e1) <= 1e-4 * np.abs(e1).max()
    assert worst(backend.download_field(d2), e2) <= 1e-4 * np.abs(e2).max()


def test_an_all_ones_mask_gives_the_unmasked_pair_bit_for_bit(backend):
    """metric/cc.rs:540-552: a mask of ones is no mask."""
    case = CASES["awkward_oblique"]
    g = fgrid(case)
    fi = backend.upload_image(g, image(case).astype(np.float32))
    mi = backend.upload_image(g, image(case, seed_offset=5).astype(np.float32))
    ones = backend.upload_image(g, np.ones(tuple(reversed(case["size"])), np.float32))
    ((a, da), (b, db)), na = backend.cc_value_derivative_pair_with_norms(fi, mi, 4)
    ((c, dc), (d, dd)), nc = backend.cc_value_derivative_pair_masked_with_norms(fi, mi, ones, 4)
    assert (a, b) == (c, d) and na == nc
    assert np.array_equal(backend.download_field(da), backend.download_field(dc))
    assert np.array_equal(backend.download_field(db), backend.download_field(dd))


def test_an_empty_mask_fails_with_no_voxel_in_masks(backend):
    """metric/cc.rs:553-565."""
    case = CASES["selftest"]
    g = fgrid(case)
    fi = backend.upload_image(g, image(case).astype(np.float32))
    zeros = backend.upload_image(g, np.zeros(tuple(reversed(case["size"])), np.float32))
    with pytest.raises(N.FastwarpError, match="no voxel of the registration level lies inside"):
        backend.cc_value_derivative_pair_masked(fi, fi, zeros, 2)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("variance", [3.0, 0.25, 8.0])
def test_smooth_field_matches(backend, name, variance):
    case = CASES[name]
    og, g = grid_of(case), fgrid(case)
    fld = field(case)
    f = backend.upload_field(g, fld)
    backend.smooth_field(f, variance)
    got = backend.download_field(f)
    want = O.smooth_field(og, fld, variance)
    assert worst(got, want) <= 2e-6 * max(1.0, np.abs(fld).max())
    same = backend.upload_field(g, fld)
    backend.smooth_field(same, 0.0)
    assert np.array_equal(backend.download_field(same), fld.astype(np.float32).astype(np.float64))


@pytest.mark.parametrize("name", NAMES)
def test_norms_scale_axpy_match(backend, name):
    case = CASES[name]
    og, g = grid_of(case), fgrid(case)
    a, b = field(case), field(case, seed_offset=33)
    fa, fb = backend.upload_field(g, a), backend.upload_field(g, b)
    assert rel(backend.max_scaled_norm(fa), O.max_scaled_norm(og, a)) <= 1e-6
    ma, mb = backend.max_scaled_norm_pair(fa, fb)
    assert rel(mb, O.max_scaled_norm(og, b)) <= 1e-6
    assert rel(backend.l2_norm(fa), O.l2_norm(og, a)) <= 1e-6
    backend.scale(fa, 0.37)
    assert worst(backend.download_field(fa), 0.37 * a) <= 1e-6 * np.abs(a).max()
    backend.axpy(fa, -2.0, fb)
    assert worst(backend.download_field(fa), 0.37 * a - 2.0 * b) <= 1e-6 * max(np.abs(a).max(), np.abs(b).max()) * 3
    c = backend.copy_field(fb)
    assert np.array_equal(backend.download_field(c), backend.download_field(fb))


@pytest.mark.parametrize("name", NAMES)
def test_compose_matches(backend, name):
    case = CASES[name]
    og, g = grid_of(case), fgrid(case)
    u, w = field(case), field(case, amp=2.5, seed_offset=9)
    out = backend.compose(backend.upload_field(g, u), backend.upload_field(g, w))
    want = O.compose(og, u, w)
    diff = np.abs(backend.download_field(out) - want).max(-1)
    # the gathered index of every voxel: x + w(x) on the same grid
    c = continuous_index(case, voxel_points(case) + w)
    assert_only_edge_flips(diff, edge_distance(case, c), 1e-5 * max(1.0, np.abs(want).max()))


@pytest.mark.parametrize("name", NAMES)
def test_invert_and_invert_pair_match(backend, name):
    case = CASES[name]
    og, g = grid_of(case), fgrid(case)
    u = field(case, amp=1.2)
    inv = backend.zero_field(g)
    _, (it, mean, mx) = backend.invert(backend.upload_field(g, u), inv)
    want, (wit, wmean, wmx) = O.invert(og, u)
    assert it == wit
    assert rel(mean, wmean) <= 1e-4 and rel(mx, wmx) <= 1e-4
    assert worst(backend.download_field(inv), want) <= 1e-4 * max(np.abs(want).max(), 1e-6)
    # the pair: inverse = invert(field, init inverse), field = invert(inverse, init field)
    f = backend.upload_field(g, u)
    i0 = backend.upload_field(g, want)
    (ri, si), (rf, sf) = backend.invert_pair(f, i0)
    wi, s1 = O.invert(og, u, want)
    wf, s2 = O.invert(og, wi, u)
    assert si[0] == s1[0] and sf[0] == s2[0]
    assert worst(backend.download_field(ri), wi) <= 1e-4 * np.abs(wi).max()
    assert worst(backend.download_field(rf), wf) <= 1e-4 * np.abs(wf).max()


def test_invert_stops_at_the_iteration_limit(backend):
    case = CASES["cube_r1"]
    og, g = grid_of(case), fgrid(case)
    u = field(case, amp=3.0)
    inv = backend.zero_field(g)
    _, (it, _, mx) = backend.invert(backend.upload_field(g, u), inv, (3, 0.0, 0.0, True))
    _, (wit, _, wmx) = O.invert(og, u, params=(3, 0.0, 0.0, True))
    assert it == wit == 3 and rel(mx, wmx) < 1e-4


@pytest.mark.parametrize("name", NAMES)
def test_resample_field_matches(backend, name):
    case = CASES[name]
    og, g = grid_of(case), fgrid(case)
    u = field(case)
    coarse = dict(case, size=tuple(max(2, s // 2) for s in case["size"]),
                  spacing=tuple(2 * s for s in case["spacing"]))
    ocg, cg = grid_of(coarse), fgrid(coarse)
    uc = field(coarse, seed_offset=3)
    got = backend.download_field(backend.resample_field(backend.upload_field(cg, uc), g))
    want = O.resample_field(ocg, uc, og)
    assert worst(got, want) <= 1e-5 * max(1.0, np.abs(want).max())


@pytest.mark.parametrize("name", ["awkward_aligned", "awkward_oblique"])
def test_recursive_gaussian_matches(backend, name):
    case = CASES[name]
    og, g = grid_of(case), fgrid(case)
    img = image(case)
    sig = (2.0 * case["spacing"][0], 2.0 * case["spacing"][1], 2.0 * case["spacing"][2])
    got = backend.smooth_recursive(backend.upload_image(g, img.astype(np.float32)), sig).download()
    want = O.smooth_recursive(og, img, sig)
    assert worst(got, want) <= 1e-5 * np.abs(want).max()


def test_closing_a_context_frees_its_buffers_first():
    from fastwarp_b200 import CudaBackend
    b = CudaBackend(0)
    g = make_grid((9, 8, 7))
    kept = [b.zero_field(g), b.upload_image(g, np.ones((7, 8, 9), np.float32))]
    b.close()
    assert all(x.handle is None for x in kept)
    del kept  # no use of the destroyed context


def test_errors_carry_the_reference_messages(backend):
    g1 = make_grid((8, 8, 8))
    g2 = make_grid((8, 8, 9))
    with pytest.raises(N.FastwarpError, match="grids differ"):
        backend.compose(backend.zero_field(g1), backend.zero_field(g2))
    with pytest.raises(N.FastwarpError, match="radius"):
        im = backend.upload_image(g1, np.zeros((8, 8, 8), np.float32))
        backend.cc_value_derivative_pair(im, im, 9)


def test_freed_buffers_are_reused_and_released_on_request(backend):
    """A context keeps the buffers it frees for the next allocation of that size (one shape
    allocates nothing after its first registration); release_idle_buffers (backend.rs:48-50)
    hands them back."""
    case = CASES["selftest"]
    g = fgrid(case)
    backend.release_idle_buffers()
    assert backend.cached_bytes() == 0
    a = backend.zero_field(g)
    a.free()
    held = backend.cached_bytes()
    assert held > 0
    b = backend.zero_field(g)  # the same size: taken from the cache
    assert backend.cached_bytes() == 0
    b.free()
    backend.release_idle_buffers()
    assert backend.cached_bytes() == 0


def test_buffers_of_sizes_no_longer_used_go_back_to_the_pool(backend):
    """A stream of requests of many grid sizes must not leave a buffer of every size in a
    context's cache: on a miss that would take the context past twice its largest working set
    (at least 1 GB), buffers idle in the cache for over a second go back to the pool; buffers
    freed more recently (the same shapes about to repeat) stay."""
    import time

    from fastwarp_b200.backend import CudaBackend

    def nbytes(n):  # a field's cached size: three planes of a 64-voxel stride, 4 KB pages
        ps = (n ** 3 + 63) // 64 * 64
        return (3 * ps * 4 + 4095) // 4096 * 4096

    with CudaBackend(backend.device) as b:  # a fresh context: its largest working set is its own
        a = b.zero_field(make_grid((292, 292, 292)))  # ~0.3 GB
        a.free()
        assert b.cached_bytes() == nbytes(292)
        time.sleep(1.2)
        c = b.zero_field(make_grid((422, 422, 422)))  # ~0.9 GB: past 1 GB with the idle buffer
        assert b.cached_bytes() == 0  # the idle buffer went back to the pool
        c.free()
        assert b.cached_bytes() == nbytes(422)
        d = b.zero_field(make_grid((322, 322, 322)))  # ~0.4 GB, at once: the 0.9 GB one stays
        assert b.cached_bytes() == nbytes(422)
        d.free()
        e = b.zero_field(make_grid((422, 422, 422)))  # the kept buffer serves the same shape
        assert b.cached_bytes() == nbytes(322)
        e.free()
