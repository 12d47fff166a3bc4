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


def grid_matrices(case):
    """(origin, index->offset matrix D diag(spacing), its inverse) of a case's grid."""
    d = np.asarray(case["direction"], float)
    ds = d * np.asarray(case["spacing"], float)[None, :]
    return np.asarray(case["origin"], float), ds, np.linalg.inv(ds)


def voxel_points(case):
    """Physical points of every voxel, shape (nz, ny, nx, 3) (grid.rs:131-140)."""
    org, ds, _ = grid_matrices(case)
    nx, ny, nz = case["size"]
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return org + np.stack([x, y, z], -1).astype(np.float64) @ ds.T


def continuous_index(case, points):
    """Continuous indices of physical points on a case's grid (grid.rs:146-156)."""
    org, _, inv = grid_matrices(case)
    return (np.asarray(points, float) - org) @ inv.T


def edge_distance(case, c):
    """Distance, in voxels, of continuous indices from the nearest buffer face (-0.5 or n - 0.5
    on any axis, where ITK's IsInsideBuffer flips)."""
    n = np.asarray(case["size"], float)
    return np.minimum(np.abs(c + 0.5), np.abs(c - (n - 0.5))).min(-1)


def vector_at(case, f, c):
    """ITK's vector linear interpolation (neighbours clamped) of an AoS field at continuous
    indices c (field_ops.rs:143-172); zero outside the buffer."""
    n = np.asarray(case["size"])
    inside = np.all((c >= -0.5) & (c < n - 0.5), -1)
    fl = np.floor(c)
    t = c - fl
    b0 = fl.astype(np.int64)
    out = np.zeros(c.shape[:-1] + (3,))
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                q = [np.clip(b0[..., a] + o, 0, n[a] - 1) for a, o in enumerate((dx, dy, dz))]
                w = np.ones(c.shape[:-1])
                for a, o in enumerate((dx, dy, dz)):
                    w = w * (t[..., a] if o else 1.0 - t[..., a])
                out += w[..., None] * f[q[2], q[1], q[0]]
    return np.where(inside[..., None], out, 0.0)
