"""Config 3: the head phantom at 0.5 mm, 385 x 457 x 385 (67.7 M voxels).

At full size the oracle cannot run a registration in test time, so the full-size run is checked
through properties that do not depend on size: each level lowers its CC energy, forward and
inverse compose to nearly the identity (syn_phantom.rs:383-512 asks < 0.25 voxel), every value is
finite and a rerun is bit-identical. Parity with the f64 oracle is checked on a crop of the same
phantom at the same spacing: one SyN CC step (1e-5 relative energy, 1e-4 voxel updates) and one
dense Mattes MI pair (1e-5 relative value, 5e-4 of the largest derivative component).

The phantom is made on the GPU with torch (test data only): nested ellipsoids 0.2/0.5/0.8 with a
degree-2 bias of +-20 % and Rician-like noise sigma 0.02, the moving image through a rigid +
affine map and a smooth displacement, as the 1 mm phantom (fastwarp_b200/phantoms.py).
"""
import numpy as np
import pytest

import oracle as O
from fastwarp_b200 import SynRecipe, make_affine, make_grid, run_syn_device, syn_step

pytestmark = pytest.mark.gpu

SHAPE = (385, 457, 385)  # x, y, z
SPACING = 0.5


def phantom_pair(shape_xyz=SHAPE, seed=20260913):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    nx, ny, nz = shape_xyz
    dev = "cuda"
    z, y, x = torch.meshgrid(*[torch.linspace(-1.0, 1.0, s, device=dev) for s in (nz, ny, nx)],
                             indexing="ij")
    img = torch.zeros((nz, ny, nx), device=dev)
    for level, (ra, rb, rc) in zip((0.2, 0.5, 0.8),
                                   [(0.85, 0.88, 0.86), (0.70, 0.74, 0.70), (0.45, 0.50, 0.42)]):
        img[(x / ra) ** 2 + (y / rb) ** 2 + (z / rc) ** 2 <= 1] = level
    for c, r, v in [((0.1, -0.2, 0.05), (0.08, 0.1, 0.07), 0.2),
                    ((-0.25, 0.15, -0.1), (0.1, 0.06, 0.09), 0.5),
                    ((0.2, 0.25, 0.2), (0.06, 0.08, 0.1), 0.2)]:
        img[((x - c[0]) / r[0]) ** 2 + ((y - c[1]) / r[1]) ** 2 + ((z - c[2]) / r[2]) ** 2 <= 1] = v
    bias = 0.6 * x + 0.3 * y - 0.4 * z + 0.5 * x * y - 0.2 * z * z
    img = img * (1.0 + 0.2 * bias / bias.abs().max())
    n1 = torch.randn(img.shape, generator=g, device=dev) * 0.02
    n2 = torch.randn(img.shape, generator=g, device=dev) * 0.02
    fixed = torch.sqrt((img + n1) ** 2 + n2 ** 2)
    # moving(q) = fixed(L^-1 (q - c) + c + u): rotation 6 deg, scale, shear, translation, smooth u
    ang = np.deg2rad([4.0, -3.0, 6.0])
    cx, sx, cy, sy, cz, sz = np.cos(ang[0]), np.sin(ang[0]), np.cos(ang[1]), np.sin(ang[1]), \
        np.cos(ang[2]), np.sin(ang[2])
    rot = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]]) @ \
        np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]]) @ \
        np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    lin = rot @ np.diag([1.04, 0.97, 1.02]) @ np.array([[1, 0.02, 0], [0, 1, -0.03], [0, 0, 1]])
    centre = np.array([(nx - 1) / 2.0, (ny - 1) / 2.0, (nz - 1) / 2.0])
    trans = np.array([6.0, -8.0, 5.0])  # voxels
    offset = centre + trans - lin @ centre
    inv = np.linalg.inv(lin)
    zi, yi, xi = torch.meshgrid(*[torch.arange(s, device=dev, dtype=torch.float32)
                                  for s in (nz, ny, nx)], indexing="ij")
    pts = torch.stack([xi, yi, zi]) - torch.tensor(offset, device=dev, dtype=torch.float32)[:, None, None, None]
    q = torch.einsum("ij,jzyx->izyx", torch.tensor(inv, device=dev, dtype=torch.float32), pts)
    u = 6.0 * torch.stack([torch.sin(2.0 * x + 0.3), torch.cos(1.5 * y - 0.2), torch.sin(1.7 * z)])
    q = q + u
    # grid_sample wants (x, y, z) in [-1, 1]
    grid = torch.stack([2 * q[0] / (nx - 1) - 1, 2 * q[1] / (ny - 1) - 1, 2 * q[2] / (nz - 1) - 1],
                       dim=-1)[None]
    moving = torch.nn.functional.grid_sample(fixed[None, None], grid, mode="bilinear",
                                             padding_mode="zeros", align_corners=True)[0, 0]
    gr = make_grid(shape_xyz, (SPACING,) * 3)
    initial = make_affine(lin, offset * SPACING)
    return gr, fixed.cpu().numpy(), moving.clamp(min=0).cpu().numpy(), initial


@pytest.fixture(scope="module")
def pair():
    return phantom_pair()


def recipe():
    return SynRecipe(gradient_step=0.1, update_field_variance=3.0, total_field_variance=0.0,
                     cc_radius=4, iterations=[40, 30, 10], shrink_factors=[4, 2, 1],
                     smoothing_sigmas=[2.0, 1.0, 0.0], convergence_threshold=-1.0,
                     convergence_window=10)


def test_full_size_registration_improves_each_level_and_is_inverse_consistent(backend, pair):
    g, fixed, moving, initial = pair
    r = recipe()
    fi, mi = backend.upload_image(g, fixed), backend.upload_image(g, moving)
    w, iw, recs = run_syn_device(backend, r, [fi], [mi], initial)
    assert len(recs) == 80
    for level in range(3):
        e = [x["energy"] for x in recs if x["level"] == level]
        assert np.isfinite(e).all()
        assert e[-1] < e[0], (level, e[0], e[-1])
    # forward o inverse: w(x) + iw(x + w(x)) ~ 0 away from the faces (half-voxel units: 0.5 mm)
    roundtrip = backend.compose(iw, w)
    a = backend.download_field(roundtrip)
    inner = a[20:-20, 20:-20, 20:-20]
    err = np.sqrt((inner ** 2).sum(-1)) / SPACING
    assert np.isfinite(a).all()
    assert err.mean() < 0.25, err.mean()
    # a rerun is bit-identical
    w2, iw2, _ = run_syn_device(backend, r, [fi], [mi], initial)
    assert np.array_equal(backend.download_field(w2), backend.download_field(w))


def crop(pair, size=(72, 80, 64)):
    g, fixed, moving, initial = pair
    nz, ny, nx = fixed.shape
    sx, sy, sz = size
    x0, y0, z0 = (nx - sx) // 2, (ny - sy) // 2 + 20, (nz - sz) // 2
    f = np.ascontiguousarray(fixed[z0:z0 + sz, y0:y0 + sy, x0:x0 + sx], dtype=np.float64)
    m = np.ascontiguousarray(moving[z0:z0 + sz, y0:y0 + sy, x0:x0 + sx], dtype=np.float64)
    return make_grid(size, (SPACING,) * 3), f, m


def test_one_cc_step_at_half_millimetre_matches_the_oracle(backend, pair):
    g, f, m = crop(pair)
    og = O.make_grid(tuple(g.size), tuple(g.spacing), tuple(g.origin))
    r = SynRecipe(gradient_step=0.1, update_field_variance=3.0, cc_radius=4, iterations=[1],
                  shrink_factors=[1], smoothing_sigmas=[0.0], convergence_threshold=-1.0)
    fi, mi = backend.upload_image(g, f), backend.upload_image(g, m)
    state = {k: backend.zero_field(g) for k in ("f2m", "f2m_inv", "m2m", "m2m_inv")}
    rec, fu, mu = syn_step(backend, r, [fi], [mi], None, state)
    shp = f.shape + (3,)
    ostate = {k: np.zeros(shp) for k in ("f2m", "f2m_inv", "m2m", "m2m_inv")}
    orec, ofu, omu = O.syn_step(O.syn_recipe(0.1, 3.0, 0.0, 4, (1,), (1,), (0.0,), False, -1.0,
                                             10, (1.0,)), og, og, [f], og, [m], None, ostate)
    assert abs(rec["energy"] - orec.energy) <= 1e-5 * abs(orec.energy)
    assert np.abs(fu - ofu).max() / SPACING <= 1e-4
    assert np.abs(mu - omu).max() / SPACING <= 1e-4


def test_one_mattes_pair_at_half_millimetre_matches_the_oracle(backend, pair):
    g, f, m = crop(pair)
    og = O.make_grid(tuple(g.size), tuple(g.spacing), tuple(g.origin))
    f32, m32 = f.astype(np.float32), m.astype(np.float32)
    fi, mi = backend.upload_image(g, f32), backend.upload_image(g, m32)
    (v0, d0), (v1, d1) = backend.mi_value_derivative_pair(fi, mi, 32)
    zero = np.zeros(f.shape + (3,))
    w0, _, e0 = O.mi_dense(og, f32.astype(np.float64), og, m32.astype(np.float64), zero, 32)
    w1, _, e1 = O.mi_dense(og, m32.astype(np.float64), og, f32.astype(np.float64), zero, 32)
    assert abs(v0 - w0) <= 1e-5 * abs(w0) and abs(v1 - w1) <= 1e-5 * abs(w1)
    assert np.abs(backend.download_field(d0) - e0).max() <= 5e-4 * np.abs(e0).max()
    assert np.abs(backend.download_field(d1) - e1).max() <= 5e-4 * np.abs(e1).max()
