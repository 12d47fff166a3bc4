"""Python mirror of the engine interface the reference's loops drive, over the C ABI.

`CudaBackend` has the operations of trait `Backend` (crates/fastwarp-reg/src/backend.rs:39-305)
under the same names and argument meanings, and `CudaLinearEngine` those of `LinearEngine` /
`LinearMetric` (crates/fastwarp-reg/src/linear.rs:288-320, optimizer.rs:60-65). Images and fields
are opaque device buffers; host arrays are numpy:

  - images: float arrays shaped (nz, ny, nx) (x fastest in memory, as `Volume`);
  - fields: float64 arrays shaped (nz, ny, nx, 3), AoS LPS millimetres (as `VectorField`).

Errors raise `FastwarpError` with the reference's message text (RegError::Invalid etc.).
"""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np

from . import _native as N
from ._native import FastwarpError, check, lib

SYN_INVERT = (20, 0.001, 0.1, True)  # InvertParams::SYN, field_ops.rs:290-295


def make_grid(size, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0), direction=None) -> N.Grid:
    """An ITK grid: size (nx, ny, nz), spacing and origin in mm, direction 3x3 (axis columns)."""
    g = N.Grid()
    d = np.eye(3) if direction is None else np.asarray(direction, dtype=np.float64)
    for a in range(3):
        g.size[a] = int(size[a])
        g.spacing[a] = float(spacing[a])
        g.origin[a] = float(origin[a])
    for k in range(9):
        g.direction[k] = float(d.reshape(-1)[k])
    return g


def grid_shape(g: N.Grid):
    return (int(g.size[2]), int(g.size[1]), int(g.size[0]))


def make_affine(matrix=None, offset=(0.0, 0.0, 0.0)) -> N.Affine:
    """y = matrix @ p + offset."""
    a = N.Affine()
    m = np.eye(3) if matrix is None else np.asarray(matrix, dtype=np.float64)
    for k in range(9):
        a.matrix[k] = float(m.reshape(-1)[k])
    for k in range(3):
        a.offset[k] = float(offset[k])
    return a


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Image:
    """An image buffer on the device (float32)."""

    def __init__(self, backend, handle):
        self.backend = backend
        self.handle = handle
        backend._live.add(self)

    @property
    def grid(self) -> N.Grid:
        g = N.Grid()
        check(lib().fw_image_grid(self.handle, C.byref(g)))
        return g

    def download(self) -> np.ndarray:
        out = np.empty(grid_shape(self.grid), np.float32)
        check(lib().fw_image_download(self.backend.ctx, self.handle, _ptr(out)))
        return out

    def free(self):
        if self.handle:
            lib().fw_image_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Field:
    """A displacement-field buffer on the device (float32 SoA planes)."""

    def __init__(self, backend, handle):
        self.backend = backend
        self.handle = handle
        backend._live.add(self)

    @property
    def grid(self) -> N.Grid:
        g = N.Grid()
        check(lib().fw_field_grid(self.handle, C.byref(g)))
        return g

    def free(self):
        if self.handle:
            lib().fw_field_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class CudaBackend:
    """trait Backend on one CUDA context (one stream; synchronous calls)."""

    def __init__(self, device: int = 0):
        ctx = C.c_void_p()
        check(lib().fw_ctx_create(int(device), C.byref(ctx)))
        self.ctx = ctx
        self.device = device
        self._live = weakref.WeakSet()  # buffers to free before the context goes

    def close(self):
        """Frees every buffer still alive on this context, then the context itself."""
        if self.ctx:
            for buf in list(self._live):
                buf.free()
            lib().fw_ctx_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def name(self) -> str:
        return lib().fw_backend_name().decode()

    def stats(self) -> dict:
        s = N.Stats()
        check(lib().fw_ctx_stats(self.ctx, C.byref(s)))
        return {k: int(getattr(s, k)) for k, _ in N.Stats._fields_}

    def release_idle_buffers(self):
        """Backend::release_idle_buffers (backend.rs:48-50): returns the buffers the context
        keeps for reuse to the device."""
        check(lib().fw_ctx_release_idle_buffers(self.ctx))

    def cached_bytes(self) -> int:
        v = C.c_uint64()
        check(lib().fw_ctx_cached_bytes(self.ctx, C.byref(v)))
        return int(v.value)

    def reset_stats(self):
        lib().fw_ctx_reset_stats(self.ctx)

    def request_cancel(self, on: bool = True) -> None:
        """fw_ctx_request_cancel: the context's own cancel flag, which the SyN level graph reads
        once per iteration (a run stops after the iteration in flight and fails with
        FW_ERR_CANCELLED). It stays set until cleared with on=False."""
        check(lib().fw_ctx_request_cancel(self.ctx, C.c_int32(1 if on else 0)))

    def synchronize(self):
        check(lib().fw_ctx_synchronize(self.ctx))

    # -- buffers (backend.rs:52-79)
    def upload_image(self, grid: N.Grid, data) -> Image:
        h = C.c_void_p()
        if isinstance(data, np.ndarray) and data.dtype == np.float32:
            a = np.ascontiguousarray(data)
            check(lib().fw_image_upload_f32(self.ctx, C.byref(grid), _ptr(a), C.byref(h)))
        else:
            a = np.ascontiguousarray(data, dtype=np.float64)
            check(lib().fw_image_upload(self.ctx, C.byref(grid), _ptr(a), C.byref(h)))
        return Image(self, h)

    def zero_field(self, grid: N.Grid) -> Field:
        h = C.c_void_p()
        check(lib().fw_field_zero(self.ctx, C.byref(grid), C.byref(h)))
        return Field(self, h)

    def upload_field(self, grid: N.Grid, data) -> Field:
        a = np.ascontiguousarray(data, dtype=np.float64)
        h = C.c_void_p()
        check(lib().fw_field_upload(self.ctx, C.byref(grid), _ptr(a), C.byref(h)))
        return Field(self, h)

    def download_field(self, field: Field) -> np.ndarray:
        out = np.empty(grid_shape(field.grid) + (3,), np.float64)
        check(lib().fw_field_download(self.ctx, field.handle, _ptr(out)))
        return out

    def field_grid(self, field: Field) -> N.Grid:
        return field.grid

    def copy_field(self, field: Field) -> Field:
        h = C.c_void_p()
        check(lib().fw_field_copy(self.ctx, field.handle, C.byref(h)))
        return Field(self, h)

    # -- operations (backend.rs:75-304)
    def warp_through_field(self, source: Image, field: Field, pre: Field | None = None,
                           affine: N.Affine | None = None) -> Image:
        h = C.c_void_p()
        check(lib().fw_warp_through_field(self.ctx, source.handle, field.handle,
                                          None if pre is None else pre.handle,
                                          None if affine is None else C.byref(affine),
                                          C.byref(h)))
        return Image(self, h)

    def warp_mask_through_field(self, mask: Image, field: Field, pre: Field | None = None,
                                affine: N.Affine | None = None,
                                product: Image | None = None) -> Image:
        h = C.c_void_p()
        check(lib().fw_warp_mask_through_field(self.ctx, mask.handle, field.handle,
                                               None if pre is None else pre.handle,
                                               None if affine is None else C.byref(affine),
                                               None if product is None else product.handle,
                                               C.byref(h)))
        if product is not None:
            return product
        return Image(self, h)

    def cc_value_derivative(self, fixed: Image, moving: Image, radius: int):
        v = C.c_double()
        h = C.c_void_p()
        check(lib().fw_cc_value_derivative(self.ctx, fixed.handle, moving.handle,
                                           C.c_int32(radius), C.byref(v), C.byref(h)))
        return v.value, Field(self, h)

    def cc_value_derivative_pair(self, fixed: Image, moving: Image, radius: int):
        vals = (C.c_double * 2)()
        a, b = C.c_void_p(), C.c_void_p()
        check(lib().fw_cc_value_derivative_pair(self.ctx, fixed.handle, moving.handle,
                                                C.c_int32(radius), vals, C.byref(a), C.byref(b)))
        return (vals[0], Field(self, a)), (vals[1], Field(self, b))

    def cc_value_derivative_pair_with_norms(self, fixed: Image, moving: Image, radius: int):
        vals = (C.c_double * 2)()
        norms = (C.c_double * 2)()
        a, b = C.c_void_p(), C.c_void_p()
        check(lib().fw_cc_value_derivative_pair_with_norms(
            self.ctx, fixed.handle, moving.handle, C.c_int32(radius), vals, C.byref(a),
            C.byref(b), norms))
        return ((vals[0], Field(self, a)), (vals[1], Field(self, b))), [norms[0], norms[1]]

    def cc_value_derivative_pair_masked(self, fixed: Image, moving: Image, valid: Image,
                                        radius: int):
        """Backend::cc_value_derivative_pair_masked (backend.rs:128-140): only voxels where
        `valid` is not zero count; raises FastwarpError naming NO_VOXEL_IN_MASKS when none does."""
        vals = (C.c_double * 2)()
        a, b = C.c_void_p(), C.c_void_p()
        check(lib().fw_cc_value_derivative_pair_masked(
            self.ctx, fixed.handle, moving.handle, valid.handle, C.c_int32(radius), vals,
            C.byref(a), C.byref(b)))
        return (vals[0], Field(self, a)), (vals[1], Field(self, b))

    def cc_value_derivative_pair_masked_with_norms(self, fixed: Image, moving: Image,
                                                   valid: Image, radius: int):
        vals = (C.c_double * 2)()
        norms = (C.c_double * 2)()
        a, b = C.c_void_p(), C.c_void_p()
        check(lib().fw_cc_value_derivative_pair_masked_with_norms(
            self.ctx, fixed.handle, moving.handle, valid.handle, C.c_int32(radius), vals,
            C.byref(a), C.byref(b), norms))
        return ((vals[0], Field(self, a)), (vals[1], Field(self, b))), [norms[0], norms[1]]

    def _mi_pair(self, fixed, moving, fixed_mask, moving_mask, bins, norms):
        vals = (C.c_double * 2)()
        nrm = (C.c_double * 2)()
        a, b = C.c_void_p(), C.c_void_p()
        fm = None if fixed_mask is None else fixed_mask.handle
        mm = None if moving_mask is None else moving_mask.handle
        check(lib().fw_mi_value_derivative_pair_masked_with_norms(
            self.ctx, fixed.handle, moving.handle, fm, mm, C.c_int32(bins), vals, C.byref(a),
            C.byref(b), nrm))
        pair = (vals[0], Field(self, a)), (vals[1], Field(self, b))
        return (pair, [nrm[0], nrm[1]]) if norms else pair

    def mi_value_derivative_pair(self, fixed: Image, moving: Image, bins: int):
        """Backend::mi_value_derivative_pair (backend.rs:179-190): dense Mattes MI both ways."""
        return self._mi_pair(fixed, moving, None, None, bins, False)

    def mi_value_derivative_pair_masked(self, fixed: Image, moving: Image, fixed_mask, moving_mask,
                                        bins: int):
        return self._mi_pair(fixed, moving, fixed_mask, moving_mask, bins, False)

    def mi_value_derivative_pair_with_norms(self, fixed: Image, moving: Image, bins: int):
        return self._mi_pair(fixed, moving, None, None, bins, True)

    def mi_value_derivative_pair_masked_with_norms(self, fixed: Image, moving: Image, fixed_mask,
                                                   moving_mask, bins: int):
        return self._mi_pair(fixed, moving, fixed_mask, moving_mask, bins, True)

    def smooth_field(self, field: Field, variance: float) -> Field:
        check(lib().fw_smooth_field(self.ctx, field.handle, C.c_double(variance)))
        return field

    def max_scaled_norm(self, field: Field) -> float:
        v = C.c_double()
        check(lib().fw_max_scaled_norm(self.ctx, field.handle, C.byref(v)))
        return v.value

    def max_scaled_norm_pair(self, a: Field, b: Field):
        out = (C.c_double * 2)()
        check(lib().fw_max_scaled_norm_pair(self.ctx, a.handle, b.handle, out))
        return out[0], out[1]

    def l2_norm(self, field: Field) -> float:
        v = C.c_double()
        check(lib().fw_l2_norm(self.ctx, field.handle, C.byref(v)))
        return v.value

    def scale(self, field: Field, s: float) -> None:
        check(lib().fw_scale(self.ctx, field.handle, C.c_double(s)))

    def axpy(self, acc: Field, a: float, x: Field) -> None:
        check(lib().fw_axpy(self.ctx, acc.handle, C.c_double(a), x.handle))

    def compose(self, displacement: Field, warping: Field) -> Field:
        h = C.c_void_p()
        check(lib().fw_compose(self.ctx, displacement.handle, warping.handle, C.byref(h)))
        return Field(self, h)

    def invert(self, field: Field, initial: Field, params=SYN_INVERT):
        prm = N.InvertParams(int(params[0]), float(params[1]), float(params[2]),
                             int(bool(params[3])))
        st = N.InvertStats()
        check(lib().fw_invert(self.ctx, field.handle, initial.handle, C.byref(prm),
                              C.byref(st)))
        return initial, (st.iterations, st.mean_error_norm, st.max_error_norm)

    def invert_pair(self, field: Field, inverse: Field, params=SYN_INVERT):
        prm = N.InvertParams(int(params[0]), float(params[1]), float(params[2]),
                             int(bool(params[3])))
        st = (N.InvertStats * 2)()
        check(lib().fw_invert_pair(self.ctx, field.handle, inverse.handle, C.byref(prm), st))
        s = [(x.iterations, x.mean_error_norm, x.max_error_norm) for x in st]
        return (inverse, s[0]), (field, s[1])

    def resample_field(self, field: Field, grid: N.Grid) -> Field:
        h = C.c_void_p()
        check(lib().fw_resample_field(self.ctx, field.handle, C.byref(grid), C.byref(h)))
        return Field(self, h)

    # -- pyramid
    def smooth_recursive(self, image: Image, sigma_mm) -> Image:
        h = C.c_void_p()
        s = (C.c_double * 3)(*[float(x) for x in sigma_mm])
        check(lib().fw_smooth_recursive(self.ctx, image.handle, s, C.byref(h)))
        return Image(self, h)

    # -- image preparation (register.rs:82-249, preprocess.rs:45-215)
    def resample_isotropic(self, image: Image, mm: float) -> Image:
        """resample_isotropic: the image on the isotropic `mm` grid (a copy if already there)."""
        h = C.c_void_p()
        check(lib().fw_resample_isotropic(self.ctx, image.handle, C.c_double(mm), C.byref(h)))
        return Image(self, h)

    def quantile_window(self, image: Image, lower: float, upper: float):
        """quantile_window: (lo, hi) of the finite voxels' 256-bin histogram, float32 values."""
        w = (C.c_double * 2)()
        check(lib().fw_quantile_window(self.ctx, image.handle, C.c_float(lower), C.c_float(upper),
                                       w))
        return w[0], w[1]

    def preprocess(self, image: Image, lower: float, upper: float, out_min: float = 0.0,
                   out_max: float = 1.0) -> Image:
        """preprocess_volume: the quantile window mapped onto [out_min, out_max]."""
        h = C.c_void_p()
        check(lib().fw_preprocess(self.ctx, image.handle, C.c_float(lower), C.c_float(upper),
                                  C.c_double(out_min), C.c_double(out_max), C.byref(h), None))
        return Image(self, h)

    def prepare_channels(self, fixed, moving, iso_mm=None, winsorize=(0.005, 0.995)):
        """prepare_channels_with: (channels as [(fixed, moving)], fixed_raw, moving_raw).
        `iso_mm` None keeps the images' grids; `winsorize` None is the plain (0, 1) rescale."""
        k = len(fixed)
        arr = C.c_void_p * max(k, 1)
        outs = [arr() for _ in range(4)]
        mm = C.byref(C.c_double(iso_mm)) if iso_mm is not None else None
        w = (C.c_float * 2)(*winsorize) if winsorize is not None else None
        check(lib().fw_prepare_channels(
            self.ctx, C.c_int32(k if k == len(moving) else 0),
            arr(*[i.handle for i in fixed]), arr(*[i.handle for i in moving]), mm, w, *outs))
        fo, mo, fr, mr = ([Image(self, C.c_void_p(o[c])) for c in range(k)] for o in outs)
        return list(zip(fo, mo)), fr, mr


def shrink_factors(factor: int, spacing):
    out = (C.c_uint32 * 3)()
    check(lib().fw_shrink_factors(C.c_uint32(factor), (C.c_double * 3)(*spacing), out))
    return tuple(out)


def shrink_grid(grid: N.Grid, factors) -> N.Grid:
    out = N.Grid()
    check(lib().fw_shrink_grid(C.byref(grid), (C.c_uint32 * 3)(*factors), C.byref(out)))
    return out


def linear_transform(kind="euler", parameters=None, center=(0, 0, 0), zyx=False,
                     outer_matrix=None, outer_translation=(0, 0, 0),
                     outer_center=(0, 0, 0)) -> N.LinearTransform:
    """LinearMovingTransform (transform/param.rs:392-420): outer(optimised(p))."""
    t = N.LinearTransform()
    om = np.eye(3) if outer_matrix is None else np.asarray(outer_matrix, np.float64)
    for k in range(9):
        t.outer_matrix[k] = float(om.reshape(-1)[k])
    for k in range(3):
        t.outer_translation[k] = float(outer_translation[k])
        t.outer_center[k] = float(outer_center[k])
        t.center[k] = float(center[k])
    t.kind = 0 if kind == "euler" else 1
    t.zyx = int(bool(zyx))
    if parameters is None:
        parameters = [0.0] * 6 if kind == "euler" else list(np.eye(3).reshape(-1)) + [0, 0, 0]
    for k, v in enumerate(parameters):
        t.parameters[k] = float(v)
    return t


def binning_from_ranges(bins, fixed_range, moving_range) -> N.MiBinning:
    """MiBinning::from_ranges (metric/mi.rs:229-262)."""
    fmin, fmax = map(float, fixed_range)
    mmin, mmax = map(float, moving_range)
    if bins <= 4:
        raise FastwarpError(N.FW_ERR_INVALID, "at least five histogram bins are required")
    if fmax - fmin <= np.finfo(np.float64).eps:
        raise FastwarpError(N.FW_ERR_INVALID, "the fixed image is constant")
    if mmax - mmin <= np.finfo(np.float64).eps:
        raise FastwarpError(N.FW_ERR_INVALID, "the moving image is constant")
    b = N.MiBinning()
    span = float(bins - 4)
    b.bins = int(bins)
    b.fixed_min, b.fixed_max, b.moving_min, b.moving_max = fmin, fmax, mmin, mmax
    b.fixed_bin_size = (fmax - fmin) / span
    b.moving_bin_size = (mmax - mmin) / span
    b.fixed_normalized_min = fmin / b.fixed_bin_size - 2.0
    b.moving_normalized_min = mmin / b.moving_bin_size - 2.0
    return b


class MiLevel:
    """LinearMetric of one prepared level (GpuMiLevel's role): -MI and its gradient."""

    def __init__(self, backend: CudaBackend, handle, keep=()):
        self.backend = backend
        self.handle = handle
        # device images the level reads in place (they must outlive it)
        self._keep = tuple(keep)
        backend._live.add(self)

    def value(self, t: N.LinearTransform) -> float:
        v = C.c_double()
        check(lib().fw_mi_level_value(self.handle, C.byref(t), C.byref(v)))
        return v.value

    def values(self, ts) -> list:
        arr = (N.LinearTransform * len(ts))(*ts)
        out = (C.c_double * len(ts))()
        check(lib().fw_mi_level_values(self.handle, arr, C.c_int32(len(ts)), out))
        return list(out)

    def value_and_derivative(self, t: N.LinearTransform):
        v = C.c_double()
        d = (C.c_double * 12)()
        check(lib().fw_mi_level_value_and_derivative(self.handle, C.byref(t), C.byref(v), d))
        n = 6 if t.kind == 0 else 12
        return v.value, np.array(d[:n])

    def time_passes(self, t: N.LinearTransform, reps: int = 20):
        """fw_mi_level_time: mean ms and algorithmic bytes per launch of the histogram pass,
        ComputeResults and the gradient pass (CUDA events on the context's stream)."""
        ms, by = (C.c_double * 3)(), (C.c_double * 3)()
        check(lib().fw_mi_level_time(self.handle, C.byref(t), C.c_int32(reps), ms, by))
        return {k: (ms[i], by[i]) for i, k in enumerate(("hist", "finish", "deriv"))}

    def samples(self):
        """fw_mi_level_samples: (points (n, 3) mm, fixed bins (n,), binning) of the level."""
        n = C.c_int64()
        b = N.MiBinning()
        check(lib().fw_mi_level_samples(self.handle, None, None, C.c_int64(0), C.byref(n),
                                        C.byref(b)))
        pts = np.empty((n.value, 3), np.float64)
        fb = np.empty(n.value, np.uint32)
        check(lib().fw_mi_level_samples(self.handle, _ptr(pts), _ptr(fb), C.c_int64(n.value),
                                        C.byref(n), None))
        return pts, fb, b

    def num_valid(self) -> int:
        v = C.c_int64()
        check(lib().fw_mi_level_num_valid(self.handle, C.byref(v)))
        return v.value

    def free(self):
        if self.handle:
            lib().fw_mi_level_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class CudaLinearEngine:
    """trait LinearEngine: prepare_level uploads the moving level image and the samples."""

    def __init__(self, backend: CudaBackend):
        self.backend = backend

    def name(self) -> str:
        return self.backend.name() + " Mattes MI"

    def prepare_level(self, moving_grid: N.Grid, moving, points, fixed_bin,
                      binning: N.MiBinning) -> MiLevel:
        m = np.ascontiguousarray(moving, np.float64)
        p = np.ascontiguousarray(points, np.float64)
        fb = np.ascontiguousarray(fixed_bin, np.uint32)
        h = C.c_void_p()
        check(lib().fw_mi_level_prepare(self.backend.ctx, C.byref(moving_grid), _ptr(m), _ptr(p),
                                        _ptr(fb), C.c_int64(p.shape[0]), C.byref(binning),
                                        C.byref(h)))
        return MiLevel(self.backend, h)

    def prepare_level_regular(self, level_grid: N.Grid, fixed: Image, moving: Image,
                              percentage: float = 0.25, seed: int = 1, bins: int = 32,
                              fixed_mask: Image | None = None) -> MiLevel:
        """The level a linear stage prepares from device images at the level's smoothing:
        regular samples of `level_grid`, their binning and fixed bins, prepared on the device
        (fw_mi_level_prepare_regular)."""
        h = C.c_void_p()
        check(lib().fw_mi_level_prepare_regular(
            self.backend.ctx, C.byref(level_grid), fixed.handle, moving.handle,
            fixed_mask.handle if fixed_mask is not None else None, C.c_float(percentage),
            C.c_uint32(seed), C.c_int32(bins), C.byref(h)))
        return MiLevel(self.backend, h, keep=(moving,))


# ---- the linear-stage optimiser (optimizer.rs:60-435) --------------------------------------------

def linear_recipe(iterations=(1000, 500, 250, 100), shrink_factors=(8, 4, 2, 1),
                  smoothing_sigmas=(3.0, 2.0, 1.0, 0.0), sigma_units_mm=False, gradient_step=0.1,
                  convergence_threshold=1e-6, convergence_window=10, bins=32,
                  sampling_percentage=0.25, seed=1) -> N.LinearRecipe:
    """LinearRecipe (linear.rs:75-128); the defaults are antsRegistration's cohort stage with the
    `MI[...,32,Regular,0.25]` metric and --random-seed 1."""
    r = N.LinearRecipe()
    r.levels = len(iterations)
    for i, (it, sf, sg) in enumerate(zip(iterations, shrink_factors, smoothing_sigmas)):
        r.iterations[i], r.shrink_factors[i], r.smoothing_sigmas[i] = int(it), int(sf), float(sg)
    r.sigma_units_mm = int(bool(sigma_units_mm))
    r.gradient_step, r.convergence_threshold = float(gradient_step), float(convergence_threshold)
    r.convergence_window, r.bins = int(convergence_window), int(bins)
    r.sampling_percentage, r.seed = float(sampling_percentage), int(seed)
    return r


def run_linear_stage(backend: "CudaBackend", recipe: N.LinearRecipe, fixed: Image,
                     moving: Image, start: N.LinearTransform, fixed_mask: Image | None = None):
    """run_linear_stage (linear.rs:512-597) on the device: (transform, [level trace dicts]).
    `fixed_mask` (an image on its own grid, non-zero inside) keeps only the sample points inside
    it (LinearRecipe::mask, linear.rs:940-945)."""
    t = N.LinearTransform.from_buffer_copy(start)
    traces = (N.LinearLevelTrace * recipe.levels)()
    check(lib().fw_linear_stage_run_masked(backend.ctx, C.byref(recipe), fixed.handle,
                                           moving.handle,
                                           fixed_mask.handle if fixed_mask is not None else None,
                                           C.byref(t), traces))
    n = 6 if t.kind == 0 else 12
    out = [dict(level=tr.level, shrink_factors=tuple(tr.shrink_factors),
                grid_size=tuple(tr.grid_size), samples=tr.samples, skipped=bool(tr.skipped),
                iterations=tr.cg.iterations, best_value=tr.cg.best_value,
                evaluations=tr.cg.line_search_evaluations, prepare_ms=tr.prepare_ms,
                optimize_ms=tr.optimize_ms, samples_cached=bool(tr.samples_cached),
                parameters=list(tr.parameters[:n])) for tr in traces]
    return t, out


def run_linear_chain(backend: "CudaBackend", rigid: N.LinearRecipe, affine: N.LinearRecipe,
                     fixed_raw: Image, moving_raw: Image, fixed: Image, moving: Image,
                     fixed_mask: Image | None = None) -> dict:
    """run_linear_chain (linear.rs:1105-1212) on the device: the centre-of-mass initial
    transform, the rigid and the affine stage, and the collapsed total, each affine transform
    as (matrix, translation, centre) with y = M (x - c) + c + t. `fixed_mask` restricts both
    stages' samples."""
    r = N.LinearChainResult()
    check(lib().fw_linear_chain_run_masked(backend.ctx, C.byref(rigid), C.byref(affine),
                                           fixed_raw.handle, moving_raw.handle, fixed.handle,
                                           moving.handle,
                                           fixed_mask.handle if fixed_mask is not None else None,
                                           C.byref(r)))

    def m3(a):
        return np.array(a[:]).reshape(3, 3)
    return {"initial": (m3(r.initial_matrix), np.array(r.initial_translation[:]),
                        np.array(r.initial_center[:])),
            "rigid": list(r.rigid.parameters[:6]), "affine": list(r.affine.parameters[:12]),
            "rigid_samples": [r.rigid_levels[k].samples for k in range(rigid.levels)],
            "affine_samples": [r.affine_levels[k].samples for k in range(affine.levels)],
            "rigid_best": [r.rigid_levels[k].cg.best_value for k in range(rigid.levels)],
            "affine_best": [r.affine_levels[k].cg.best_value for k in range(affine.levels)],
            "rigid_iterations": [r.rigid_levels[k].cg.iterations for k in range(rigid.levels)],
            "affine_iterations": [r.affine_levels[k].cg.iterations for k in range(affine.levels)],
            "rigid_evaluations": [r.rigid_levels[k].cg.line_search_evaluations
                                  for k in range(rigid.levels)],
            "affine_evaluations": [r.affine_levels[k].cg.line_search_evaluations
                                   for k in range(affine.levels)],
            "rigid_prepare_ms": [r.rigid_levels[k].prepare_ms for k in range(rigid.levels)],
            "affine_prepare_ms": [r.affine_levels[k].prepare_ms for k in range(affine.levels)],
            "rigid_optimize_ms": [r.rigid_levels[k].optimize_ms for k in range(rigid.levels)],
            "affine_optimize_ms": [r.affine_levels[k].optimize_ms for k in range(affine.levels)],
            "affine_samples_cached": [bool(r.affine_levels[k].samples_cached)
                                      for k in range(affine.levels)],
            "initial_ms": r.initial_ms,
            "total": (m3(r.total_matrix), np.array(r.total_translation[:]),
                      np.array(r.total_center[:])),
            # each stage's whole transform (the earlier transforms as its outer part)
            "rigid_transform": N.LinearTransform.from_buffer_copy(r.rigid),
            "affine_transform": N.LinearTransform.from_buffer_copy(r.affine)}


def cg_settings_ants(max_step_mm=0.1, iterations=100, threshold=1e-6, window=10) -> N.CgSettings:
    """CgSettings::ants (optimizer.rs:94-106)."""
    s = N.CgSettings()
    lib().fw_cg_settings_ants(C.c_double(max_step_mm), C.c_int32(iterations),
                              C.c_double(threshold), C.c_int32(window), C.byref(s))
    return s


def grid_corners(grid: N.Grid) -> np.ndarray:
    """corner_points (optimizer.rs:142-166): (8, 3) physical corner points."""
    out = (C.c_double * 24)()
    check(lib().fw_grid_corners(C.byref(grid), out))
    return np.array(out[:]).reshape(8, 3)


def _trace(tr: N.CgTrace, values, n_params) -> dict:
    return {"iterations": tr.iterations, "converged": bool(tr.converged),
            "converged_value": None if np.isnan(tr.converged_value) else tr.converged_value,
            "best_value": tr.best_value, "initial_learning_rate": tr.initial_learning_rate,
            "final_learning_rate": tr.final_learning_rate,
            "line_search_evaluations": tr.line_search_evaluations,
            "scales": list(tr.scales[:n_params]), "values": list(values[:min(tr.nvalues, len(values))])}


def optimize_level(value, value_and_derivative, corners, transform: N.LinearTransform,
                   settings: N.CgSettings, cap: int = 100000):
    """optimise_level (optimizer.rs:311-435) over a Python metric: `value(t) -> float` and
    `value_and_derivative(t) -> (float, derivative)`. Returns (best transform, trace)."""
    nparams = 6 if transform.kind == 0 else 12
    err = []

    def v_cb(user, t, out):
        try:
            out[0] = float(value(t.contents))
            return 0
        except Exception as e:  # reported through the optimiser's error
            err.append(e)
            return -1

    def vd_cb(user, t, out, d):
        try:
            val, der = value_and_derivative(t.contents)
            out[0] = float(val)
            for i in range(nparams):
                d[i] = float(der[i])
            return 0
        except Exception as e:
            err.append(e)
            return -1

    c = (C.c_double * 24)(*np.asarray(corners, np.float64).ravel())
    t = N.LinearTransform.from_buffer_copy(transform)
    tr = N.CgTrace()
    vals = (C.c_double * cap)()
    f1, f2 = N.METRIC_VALUE_FN(v_cb), N.METRIC_VALUE_DERIVATIVE_FN(vd_cb)
    rc = lib().fw_cg_optimize_level(C.byref(settings), c, C.byref(t), f1, f2, None,
                                    C.byref(tr), vals, C.c_int64(cap), None)
    if err:
        raise err[0]
    check(rc)
    return t, _trace(tr, vals, nparams)


def mi_level_optimize(level, corners, transform: N.LinearTransform, settings: N.CgSettings,
                      cap: int = 100000):
    """The optimiser on a device MI level (fw_mi_level_optimize)."""
    nparams = 6 if transform.kind == 0 else 12
    c = (C.c_double * 24)(*np.asarray(corners, np.float64).ravel())
    t = N.LinearTransform.from_buffer_copy(transform)
    tr = N.CgTrace()
    vals = (C.c_double * cap)()
    check(lib().fw_mi_level_optimize(level.handle, C.byref(settings), c, C.byref(t), C.byref(tr),
                                     vals, C.c_int64(cap)))
    return t, _trace(tr, vals, nparams)
