"""Seeded synthetic image pairs with the shapes and value distributions of the benchmark configs.

No public dataset is used: every pair is generated from a seed (base 20 260 910, the cohort seed
of the reference's linear recipe, plus the config index). Images are float32 (nz, ny, nx) on 1 mm
isotropic grids with identity direction.

  - `blob_pair` (64^3): 12 anisotropic Gaussian blobs (centres uniform in the inner 80 %, sigma
    U(3, 10) voxels per axis, amplitude U(0.3, 1.0)) normalised to [0, 1]; the moving image is
    the fixed image warped by a random smooth field (N(0, 1) per component, Gaussian sigma 6
    voxels, rescaled to max |u| = 3 voxels) plus N(0, 0.01) noise.
  - `head_pair` (193 x 229 x 193): nested ellipsoids with classes 0.2 / 0.5 / 0.8, a degree-2
    multiplicative bias (+-20 %) and Rician-like noise sigma 0.02; the moving image is the fixed
    image under a random rigid (<= 10 deg per axis, <= 15 mm), affine (scale 0.9-1.1, shear
    <= 0.05) and smooth displacement (<= 6 mm) map. The linear part is returned as the SyN stage's
    initial transform (fixed points to moving points).
"""
from __future__ import annotations

import numpy as np

from .backend import make_affine, make_grid

BASE_SEED = 20_260_910


def _gaussian(a, sigma):
    from scipy.ndimage import gaussian_filter
    return gaussian_filter(a, sigma, mode="nearest")


def _warp(img, coords):
    from scipy.ndimage import map_coordinates
    return map_coordinates(img, coords, order=1, mode="nearest")


def _smooth_field(rng, shape, sigma, max_norm, coarse=1):
    """Three smoothed N(0,1) components rescaled so the largest vector norm is max_norm."""
    from scipy.ndimage import zoom
    cshape = tuple(max(4, s // coarse) for s in shape)
    comps = []
    for _ in range(3):
        c = _gaussian(rng.standard_normal(cshape), sigma / coarse)
        if coarse > 1:
            c = zoom(c, [s / cs for s, cs in zip(shape, cshape)], order=1)
        comps.append(c)
    u = np.stack(comps)
    scale = max_norm / np.sqrt((u ** 2).sum(0)).max()
    return u * scale


def blob_pair(n: int = 64, seed: int = BASE_SEED + 1):
    """Config 1: (grid, fixed, moving) float32 (n, n, n)."""
    rng = np.random.default_rng(seed)
    shape = (n, n, n)
    zz, yy, xx = np.meshgrid(*[np.arange(s, dtype=np.float64) for s in shape], indexing="ij")
    img = np.zeros(shape)
    for _ in range(12):
        c = rng.uniform(0.1 * n, 0.9 * n, size=3)
        s = rng.uniform(3.0, 10.0, size=3)
        a = rng.uniform(0.3, 1.0)
        img += a * np.exp(-0.5 * (((xx - c[0]) / s[0]) ** 2 + ((yy - c[1]) / s[1]) ** 2 +
                                  ((zz - c[2]) / s[2]) ** 2))
    img = (img - img.min()) / (img.max() - img.min())
    u = _smooth_field(rng, shape, 6.0, 3.0)  # components ordered (z, y, x) offsets
    moving = _warp(img, np.stack([zz + u[0], yy + u[1], xx + u[2]]))
    moving = moving + rng.normal(0.0, 0.01, size=shape)
    grid = make_grid((n, n, n))
    return grid, img.astype(np.float32), moving.astype(np.float32)


def _rot(ax, ay, az):
    cx, sx, cy, sy, cz, sz = np.cos(ax), np.sin(ax), np.cos(ay), np.sin(ay), np.cos(az), np.sin(az)
    rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return rz @ rx @ ry


def head_phantom(shape_xyz=(193, 229, 193), seed: int = BASE_SEED + 2):
    """The fixed image of config 2: float32 (nz, ny, nx)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape_xyz
    shape = (nz, ny, nx)
    zz, yy, xx = np.meshgrid(*[np.linspace(-1.0, 1.0, s) for s in shape], indexing="ij")
    img = np.zeros(shape, np.float64)
    radii = [(0.85, 0.88, 0.86), (0.70, 0.74, 0.70), (0.45, 0.50, 0.42)]
    for level, (ra, rb, rc) in zip((0.2, 0.5, 0.8), radii):
        jit = rng.uniform(-0.03, 0.03, size=3)
        inside = ((xx - jit[0]) / ra) ** 2 + ((yy - jit[1]) / rb) ** 2 + ((zz - jit[2]) / rc) ** 2 <= 1
        img[inside] = level
    # small inner structures so the interior is not flat
    for _ in range(6):
        c = rng.uniform(-0.35, 0.35, size=3)
        r = rng.uniform(0.05, 0.12, size=3)
        inside = ((xx - c[0]) / r[0]) ** 2 + ((yy - c[1]) / r[1]) ** 2 + ((zz - c[2]) / r[2]) ** 2 <= 1
        img[inside] = rng.choice([0.2, 0.5])
    # degree-2 multiplicative bias, +-20 %
    coef = rng.uniform(-1.0, 1.0, size=10)
    terms = [np.ones_like(xx), xx, yy, zz, xx * xx, yy * yy, zz * zz, xx * yy, yy * zz, xx * zz]
    bias = sum(c * t for c, t in zip(coef, terms))
    bias = 0.2 * bias / np.abs(bias).max()
    img = img * (1.0 + bias)
    n1 = rng.normal(0.0, 0.02, size=shape)
    n2 = rng.normal(0.0, 0.02, size=shape)
    img = np.sqrt((img + n1) ** 2 + n2 ** 2)
    return img.astype(np.float32)


def head_pair(shape_xyz=(193, 229, 193), seed: int = BASE_SEED + 2, spacing: float = 1.0):
    """Config 2: (grid, fixed, moving_grid, moving, initial affine). With spacing 0.5 and twice
    the shape, config 3: the same head geometry sampled finer, with fresh noise per voxel."""
    rng = np.random.default_rng(seed + 1000)
    fixed = head_phantom(shape_xyz, seed)
    nx, ny, nz = shape_xyz
    grid = make_grid(shape_xyz, (spacing,) * 3)
    centre = np.array([(nx - 1) / 2.0, (ny - 1) / 2.0, (nz - 1) / 2.0])
    rot = _rot(*np.deg2rad(rng.uniform(-10.0, 10.0, size=3)))
    trans = rng.uniform(-15.0, 15.0, size=3)
    scale = np.diag(rng.uniform(0.9, 1.1, size=3))
    shear = np.eye(3)
    shear[0, 1], shear[0, 2], shear[1, 2] = rng.uniform(-0.05, 0.05, size=3)
    lin = rot @ scale @ shear
    # fixed points to moving points: y = lin (x - c) + c + t
    offset = centre + trans - lin @ centre
    # moving(y) = fixed(psi(y)), psi(y) = L^-1(y) + u(L^-1 y): a smooth deformation in fixed space
    shape = (nz, ny, nx)
    u = _smooth_field(rng, shape, 12.0, 6.0, coarse=4)
    zz, yy, xx = np.meshgrid(*[np.arange(s, dtype=np.float64) for s in shape], indexing="ij")
    pts = np.stack([xx.ravel(), yy.ravel(), zz.ravel()])
    inv = np.linalg.inv(lin)
    q = inv @ (pts - offset[:, None])
    qx, qy, qz = (q[0].reshape(shape), q[1].reshape(shape), q[2].reshape(shape))
    coords = np.stack([qz, qy, qx])
    ux = _warp(u[2], coords)
    uy = _warp(u[1], coords)
    uz = _warp(u[0], coords)
    moving = _warp(fixed.astype(np.float64), np.stack([qz + uz, qy + uy, qx + ux]))
    moving = np.clip(moving, 0.0, None).astype(np.float32)
    # index-space map -> physical: isotropic spacing scales the offset only
    initial = make_affine(lin, offset * spacing)
    return grid, fixed, grid, moving, initial


def t2_like(t1):
    """The T2w-like channel of config 4: inverted tissue contrast inside the head (1 - value where
    the T1-like value exceeds the background), background unchanged."""
    head = t1 > 0.1
    return np.where(head, 1.0 - t1, t1).astype(np.float32)


def batch_subjects(backend, n, template_shape=(193, 229, 193), dims=(160, 240),
                   seed: int = BASE_SEED + 4):
    """Config 4 on the device: the template's two channels (the head phantom as the T1-like one
    and its inverted-contrast T2-like copy) and `n` subjects, each on its own 1 mm grid with dims
    drawn uniformly per axis from `dims`, made from the template by an independent random rigid
    (<= 10 deg, <= 15 mm) and affine (scale 0.9-1.1, shear <= 0.05) map and a smooth displacement
    (<= 6 mm), warped on the device (subject(x) = template(A(x + u(x))) for every channel).
    Returns (template grid, [t1, t2] device images, [([s1, s2] device images, initial affine)]):
    the initial affine maps template points to subject points (the linear part of A, inverted),
    as a converged linear stage would."""
    rng = np.random.default_rng(seed)
    t1 = head_phantom(template_shape, seed)
    g = make_grid(template_shape)
    imgs = [backend.upload_image(g, t1), backend.upload_image(g, t2_like(t1))]
    ct = (np.array(template_shape, float) - 1.0) / 2.0
    subjects = []
    for _ in range(n):
        d = np.array([int(rng.integers(dims[0], dims[1] + 1)) for _ in range(3)])
        cs = (d - 1.0) / 2.0
        origin = ct - cs + rng.uniform(-5.0, 5.0, size=3)
        sg = make_grid(tuple(int(x) for x in d), (1.0, 1.0, 1.0), tuple(origin))
        rot = _rot(*np.deg2rad(rng.uniform(-10.0, 10.0, size=3)))
        scale = np.diag(rng.uniform(0.9, 1.1, size=3))
        shear = np.eye(3)
        shear[0, 1], shear[0, 2], shear[1, 2] = rng.uniform(-0.05, 0.05, size=3)
        lin = rot @ scale @ shear
        centre_s = origin + cs
        # subject points to template points: p_t = lin (p_s - centre_s) + ct + t
        off = ct + rng.uniform(-15.0, 15.0, size=3) - lin @ centre_s
        # a smooth displacement on the subject grid: components on a grid 4x coarser, upsampled
        cd = tuple(int(x) for x in np.maximum(4, np.ceil(d / 4.0)))
        comps = [_gaussian(rng.standard_normal(cd[::-1]), 3.0) for _ in range(3)]
        u = np.stack(comps, -1)
        u *= 6.0 / np.sqrt((u ** 2).sum(-1)).max()
        cg = make_grid(cd, (4.0, 4.0, 4.0), tuple(origin + 1.5))
        field = backend.resample_field(backend.upload_field(cg, u), sg)
        A = make_affine(lin, off)
        moving = [backend.warp_through_field(im, field, affine=A) for im in imgs]
        inv = np.linalg.inv(lin)
        initial = make_affine(inv, -inv @ off)
        subjects.append((moving, initial))
    return g, imgs, subjects


def _random_linear(rng):
    """Config 2's random linear part: rigid (<= 10 deg per axis) then affine (scale 0.9-1.1,
    shear <= 0.05)."""
    rot = _rot(*np.deg2rad(rng.uniform(-10.0, 10.0, size=3)))
    scale = np.diag(rng.uniform(0.9, 1.1, size=3))
    shear = np.eye(3)
    shear[0, 1], shear[0, 2], shear[1, 2] = rng.uniform(-0.05, 0.05, size=3)
    return rot @ scale @ shear


def _device_field(backend, rng, grid, d, origin, max_mm=6.0):
    """A smooth displacement (<= max_mm) on `grid`: components on a grid 4x coarser, upsampled."""
    cd = tuple(int(x) for x in np.maximum(4, np.ceil(np.asarray(d) / 4.0)))
    u = np.stack([_gaussian(rng.standard_normal(cd[::-1]), 3.0) for _ in range(3)], -1)
    u *= max_mm / np.sqrt((u ** 2).sum(-1)).max()
    cg = make_grid(cd, (4.0, 4.0, 4.0), tuple(np.asarray(origin) + 1.5))
    return backend.resample_field(backend.upload_field(cg, u), grid)


def stream_requests(backend, n, mix=(0.7, 0.2, 0.1), dims=(160, 240), template_shape=(193, 229, 193),
                    seed: int = BASE_SEED + 5):
    """Config 5's requests on the device: `n` seeded phantom pairs, each on its own 1 mm grid of
    dims drawn uniformly per axis from `dims`; the kind is drawn from `mix` over ("syn" single
    channel, "affine" an affine-only Mattes MI fit, "syn2" two channels). As in config 2 the fixed
    image is the head phantom (placed on the request's grid with a shift of up to 5 mm) and the
    moving image the fixed image under a random rigid + affine map and a smooth displacement
    (<= 6 mm), on the same grid; the linear part is the SyN requests' initial transform. Returns
    dicts: kind, grid, fixed / moving ([device image per channel]), initial (affine, fixed
    points to moving points)."""
    rng = np.random.default_rng(seed)
    t1 = head_phantom(template_shape, seed)
    tg = make_grid(template_shape)
    tmpl = [backend.upload_image(tg, t1), backend.upload_image(tg, t2_like(t1))]
    ct = (np.array(template_shape, float) - 1.0) / 2.0
    kinds = ("syn", "affine", "syn2")
    out = []
    for _ in range(n):
        kind = kinds[int(rng.choice(3, p=np.asarray(mix) / np.sum(mix)))]
        d = np.array([int(rng.integers(dims[0], dims[1] + 1)) for _ in range(3)])
        cs = (d - 1.0) / 2.0
        origin = ct - cs
        g = make_grid(tuple(int(x) for x in d), (1.0, 1.0, 1.0), tuple(origin))
        zero = backend.zero_field(g)
        shift = make_affine(np.eye(3), rng.uniform(-5.0, 5.0, size=3))
        chans = 2 if kind == "syn2" else 1
        fixed = [backend.warp_through_field(tmpl[c], zero, affine=shift) for c in range(chans)]
        lin = _random_linear(rng)
        centre = origin + cs
        off = centre + rng.uniform(-15.0, 15.0, size=3) - lin @ centre
        u = _device_field(backend, rng, g, d, origin)
        # moving(y) = fixed(A(y + u(y))): A maps moving points to fixed points
        moving = [backend.warp_through_field(f, u, affine=make_affine(lin, off)) for f in fixed]
        inv = np.linalg.inv(lin)
        out.append({"kind": kind, "grid": g, "fixed": fixed, "moving": moving,
                    "initial": make_affine(inv, -inv @ off)})
    return out
