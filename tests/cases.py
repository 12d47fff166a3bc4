"""Parity cases in the style of the reference's harness (crates/fastwarp-gpu/src/parity.rs:60-128):
odd sizes, anisotropic spacing, oblique directions, seeded smooth content."""
import numpy as np

import oracle as O


def rot_z(a):
    c, s = np.cos(a), np.sin(a)
    return np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])


def rot_x(a):
    c, s = np.cos(a), np.sin(a)
    return np.array([[1.0, 0.0, 0.0], [0.0, c, -s], [0.0, s, c]])


CASES = {
    # parity.rs:89-99 Case::selftest
    "selftest": dict(size=(11, 9, 8), spacing=(1.5, 2.0, 1.25), origin=(-8.0, 5.0, -3.5),
                     direction=rot_z(0.3) @ rot_x(0.2), radius=2, seed=7),
    # Case::awkward shapes: oblique and axis-aligned
    "awkward_oblique": dict(size=(37, 29, 23), spacing=(1.1, 0.9, 1.3), origin=(-12.5, 7.25, -4.0),
                            direction=rot_z(-0.41) @ rot_x(0.27), radius=4, seed=11),
    "awkward_aligned": dict(size=(41, 33, 27), spacing=(1.0, 1.5, 0.75), origin=(-12.5, 7.25, -4.0),
                            direction=np.eye(3), radius=3, seed=13),
    "long_thin": dict(size=(97, 7, 5), spacing=(0.8, 1.2, 1.0), origin=(3.0, -2.0, 1.0),
                      direction=np.eye(3), radius=2, seed=17),
    "cube_r1": dict(size=(24, 24, 24), spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0),
                    direction=np.eye(3), radius=1, seed=19),
}


def grid_of(case):
    return O.make_grid(case["size"], case["spacing"], case["origin"], case["direction"])


def image(case, seed_offset=0, noise=0.02):
    """Smooth seeded content in [0, ~1.5] plus a little noise, shape (nz, ny, nx)."""
    rng = np.random.default_rng(case["seed"] + seed_offset)
    nx, ny, nz = case["size"]
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    img = np.zeros((nz, ny, nx))
    for _ in range(4):
        k = rng.uniform(0.15, 0.5, size=3)
        ph = rng.uniform(0, 2 * np.pi, size=3)
        img += rng.uniform(0.1, 0.3) * (np.sin(k[0] * x + ph[0]) * np.cos(k[1] * y + ph[1]) +
                                        np.sin(k[2] * z + ph[2]))
    img = img - img.min()
    img += noise * rng.standard_normal(img.shape)
    return img.astype(np.float32).astype(np.float64)


def field(case, amp=1.5, seed_offset=100):
    """A smooth displacement field (nz, ny, nx, 3) in mm, float32-representable."""
    rng = np.random.default_rng(case["seed"] + seed_offset)
    nx, ny, nz = case["size"]
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    out = np.zeros((nz, ny, nx, 3))
    for c in range(3):
        k = rng.uniform(0.1, 0.35, size=3)
        ph = rng.uniform(0, 2 * np.pi, size=3)
        out[..., c] = amp * np.sin(k[0] * x + ph[0]) * np.sin(k[1] * y + ph[1]) * np.cos(k[2] * z + ph[2])
    return out.astype(np.float32).astype(np.float64)


def interior(shape, margin=1):
    """Mask of voxels at least `margin` voxels inside every face."""
    m = np.zeros(shape, bool)
    m[margin:shape[0] - margin, margin:shape[1] - margin, margin:shape[2] - margin] = True
    return m
