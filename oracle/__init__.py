"""CPU oracle of the fastwarp registration hot path (ctypes wrapper of ``libfw_oracle.so``).

TEST INFRASTRUCTURE ONLY: this package is the parity checker used by ``tests/`` and the timed
CPU baseline of ``bench.py``. The product (``fastwarp_b200``) never imports it.

The library is an f64 OpenMP restatement of the reference's CPU engine (crate fastwarp-reg of
WyssCenter/fastwarp); ``fw_oracle.cpp`` cites the reference file:line beside every function.
Images are float64 arrays shaped ``(nz, ny, nx)`` (x fastest in memory, as the reference);
fields are float64 arrays shaped ``(nz, ny, nx, 3)`` (AoS millimetre displacements).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libfw_oracle.so")


class Grid(C.Structure):
    _fields_ = [("size", C.c_int64 * 3), ("spacing", C.c_double * 3),
                ("origin", C.c_double * 3), ("direction", C.c_double * 9)]


class Affine(C.Structure):
    _fields_ = [("matrix", C.c_double * 9), ("offset", C.c_double * 3)]


class InvertParams(C.Structure):
    _fields_ = [("max_iterations", C.c_int32), ("mean_error_tolerance", C.c_double),
                ("max_error_tolerance", C.c_double), ("enforce_boundary_condition", C.c_int32)]


class InvertStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("mean_error_norm", C.c_double),
                ("max_error_norm", C.c_double)]


class MiBinning(C.Structure):
    _fields_ = [("bins", C.c_int32), ("fixed_min", C.c_double), ("fixed_max", C.c_double),
                ("moving_min", C.c_double), ("moving_max", C.c_double),
                ("fixed_bin_size", C.c_double), ("moving_bin_size", C.c_double),
                ("fixed_normalized_min", C.c_double), ("moving_normalized_min", C.c_double)]


class LinearTransform(C.Structure):
    _fields_ = [("outer_matrix", C.c_double * 9), ("outer_translation", C.c_double * 3),
                ("outer_center", C.c_double * 3), ("kind", C.c_int32), ("zyx", C.c_int32),
                ("parameters", C.c_double * 12), ("center", C.c_double * 3)]


MAX_LEVELS = 8
MAX_CHANNELS = 4


class SynRecipe(C.Structure):
    _fields_ = [("gradient_step", C.c_double), ("update_field_variance", C.c_double),
                ("total_field_variance", C.c_double), ("cc_radius", C.c_int32),
                ("levels", C.c_int32), ("iterations", C.c_uint32 * MAX_LEVELS),
                ("shrink_factors", C.c_uint32 * MAX_LEVELS),
                ("smoothing_sigmas", C.c_double * MAX_LEVELS), ("sigma_units_mm", C.c_int32),
                ("convergence_threshold", C.c_double), ("convergence_window", C.c_int32),
                ("channels", C.c_int32), ("channel_weights", C.c_double * MAX_CHANNELS),
                ("channel_metrics", C.c_int32 * MAX_CHANNELS), ("mi_bins", C.c_int32)]


class SynIteration(C.Structure):
    _fields_ = [("level", C.c_int32), ("energy", C.c_double), ("energy_weighted", C.c_double),
                ("convergence_value", C.c_double), ("fixed_update_scale", C.c_double),
                ("moving_update_scale", C.c_double), ("inversions", InvertStats * 4)]


SYN_INVERT = (20, 0.001, 0.1, True)

_lib = None


def build() -> None:
    """Compiles the oracle library with its Makefile (g++, OpenMP)."""
    subprocess.run(["make", "-C", _HERE], check=True, capture_output=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _lib.fwo_last_error.restype = C.c_char_p
        for name in ("fwo_max_scaled_norm", "fwo_l2_norm", "fwo_bspline3",
                     "fwo_bspline3_derivative", "fwo_convergence_value"):
            getattr(_lib, name).restype = C.c_double
        _lib.fwo_gaussian_taps.restype = C.c_int64
        _lib.fwo_sample_points_regular.restype = C.c_int64
        _lib.fwo_convergence_value.argtypes = [C.c_void_p, C.c_int64, C.c_int32, C.c_double]
        _lib.fwo_bspline3.argtypes = [C.c_double]
        _lib.fwo_bspline3_derivative.argtypes = [C.c_double]
        _lib.fwo_gaussian_taps.argtypes = [C.c_double, C.c_double, C.c_int64, C.c_void_p,
                                           C.c_int64]
        _lib.fwo_sample_points_regular.argtypes = [C.c_void_p, C.c_float, C.c_uint32,
                                                   C.c_void_p, C.c_int64]
    return _lib


class OracleError(RuntimeError):
    pass


def _check(rc):
    if rc != 0:
        raise OracleError(lib().fwo_last_error().decode())


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def set_threads(n: int) -> None:
    lib().fwo_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().fwo_num_threads())


def make_grid(size, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0), direction=None) -> Grid:
    """size is (nx, ny, nz); direction is a 3x3 (row-major, columns are the axis directions)."""
    g = Grid()
    for a in range(3):
        g.size[a] = int(size[a])
        g.spacing[a] = float(spacing[a])
        g.origin[a] = float(origin[a])
    d = np.eye(3) if direction is None else np.asarray(direction, dtype=np.float64)
    for k in range(9):
        g.direction[k] = float(d.reshape(-1)[k])
    return g


def grid_shape(g: Grid):
    return (g.size[2], g.size[1], g.size[0])


def make_affine(matrix=None, offset=(0.0, 0.0, 0.0)) -> Affine:
    a = Affine()
    m = np.eye(3) if matrix is None else np.asarray(matrix, dtype=np.float64)
    for k in range(9):
        a.matrix[k] = float(m.reshape(-1)[k])
    for k in range(3):
        a.offset[k] = float(offset[k])
    return a


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def warp(src_grid, src, grid, field, pre_grid=None, pre=None, affine=None):
    out = np.empty(grid_shape(grid), np.float64)
    src, field = _f64(src), _f64(field)
    pre = None if pre is None else _f64(pre)
    _check(lib().fwo_warp(C.byref(src_grid), _p(src), C.byref(grid), _p(field),
                          None if pre_grid is None else C.byref(pre_grid), _p(pre),
                          None if affine is None else C.byref(affine), _p(out)))
    return out


def warp_mask(mask_grid, mask, grid, field, pre_grid=None, pre=None, affine=None, product=None):
    out = np.empty(grid_shape(grid), np.float64)
    mask, field = _f64(mask), _f64(field)
    pre = None if pre is None else _f64(pre)
    product = None if product is None else _f64(product)
    _check(lib().fwo_warp_mask(C.byref(mask_grid), _p(mask), C.byref(grid), _p(field),
                               None if pre_grid is None else C.byref(pre_grid), _p(pre),
                               None if affine is None else C.byref(affine), _p(product),
                               _p(out)))
    return out


def cc(grid, fixed, moving, radius, valid=None, derivative=True):
    """One CC evaluation: (value, derivative, local_cc, coefficient, num_valid)."""
    fixed, moving = _f64(fixed), _f64(moving)
    valid = None if valid is None else _f64(valid)
    shape = grid_shape(grid)
    d = np.zeros(shape + (3,)) if derivative else None
    lcc = np.zeros(shape)
    coeff = np.zeros(shape)
    value = C.c_double()
    nv = C.c_int64()
    _check(lib().fwo_cc(C.byref(grid), _p(fixed), _p(moving), _p(valid), C.c_int32(radius),
                        C.byref(value), _p(d), _p(lcc), _p(coeff), C.byref(nv)))
    return value.value, d, lcc, coeff, nv.value


def cc_pair(grid, fixed, moving, radius, valid=None):
    fixed, moving = _f64(fixed), _f64(moving)
    valid = None if valid is None else _f64(valid)
    shape = grid_shape(grid) + (3,)
    d1, d2 = np.zeros(shape), np.zeros(shape)
    vals = (C.c_double * 2)()
    _check(lib().fwo_cc_pair(C.byref(grid), _p(fixed), _p(moving), _p(valid), C.c_int32(radius),
                             vals, _p(d1), _p(d2)))
    return (vals[0], d1), (vals[1], d2)


def gaussian_taps(variance, max_error=0.001, max_width=1000):
    out = np.zeros(4096)
    n = lib().fwo_gaussian_taps(variance, max_error, max_width, _p(out), 4096)
    return out[:n].copy()


def smooth_field(grid, field, variance):
    field = _f64(field)
    out = np.empty_like(field)
    _check(lib().fwo_smooth_field(C.byref(grid), _p(field), C.c_double(variance), _p(out)))
    return out


def max_scaled_norm(grid, field):
    lib().fwo_max_scaled_norm.argtypes = [C.c_void_p, C.c_void_p]
    return lib().fwo_max_scaled_norm(C.byref(grid), _p(_f64(field)))


def l2_norm(grid, field):
    return lib().fwo_l2_norm(C.byref(grid), _p(_f64(field)))


def compose(grid, displacement, warping):
    d, w = _f64(displacement), _f64(warping)
    out = np.empty_like(w)
    _check(lib().fwo_compose(C.byref(grid), _p(d), _p(w), _p(out)))
    return out


def invert(grid, field, initial=None, params=SYN_INVERT):
    field = _f64(field)
    inv = np.zeros_like(field) if initial is None else _f64(initial).copy()
    prm = InvertParams(int(params[0]), float(params[1]), float(params[2]), int(bool(params[3])))
    st = InvertStats()
    _check(lib().fwo_invert(C.byref(grid), _p(field), _p(inv), C.byref(prm), C.byref(st)))
    return inv, (st.iterations, st.mean_error_norm, st.max_error_norm)


def resample_field(src_grid, field, grid):
    field = _f64(field)
    out = np.empty(grid_shape(grid) + (3,), np.float64)
    _check(lib().fwo_resample_field(C.byref(src_grid), _p(field), C.byref(grid), _p(out)))
    return out


def smooth_recursive(grid, img, sigma_mm):
    img = _f64(img)
    out = np.empty_like(img)
    s = (C.c_double * 3)(*[float(x) for x in sigma_mm])
    _check(lib().fwo_smooth_recursive(C.byref(grid), _p(img), s, _p(out)))
    return out


def shrink_factors(factor, spacing):
    out = (C.c_uint32 * 3)()
    lib().fwo_shrink_factors(C.c_uint32(factor), (C.c_double * 3)(*spacing), out)
    return tuple(out)


def shrink_grid(grid, factors):
    out = Grid()
    _check(lib().fwo_shrink_grid(C.byref(grid), (C.c_uint32 * 3)(*factors), C.byref(out)))
    return out


def quantile_window(values, lower, upper):
    """preprocess.rs:168-173: (lo, hi), each rounded to float32."""
    v = _f64(np.ravel(values))
    out = (C.c_double * 2)()
    _check(lib().fwo_quantile_window(_p(v), C.c_int64(v.size), C.c_float(lower),
                                     C.c_float(upper), out))
    return out[0], out[1]


def preprocess(values, lower, upper, out_min=0.0, out_max=1.0):
    """preprocess.rs:180-209: the quantile window mapped onto [out_min, out_max]."""
    v = _f64(values)
    out = np.empty_like(v)
    _check(lib().fwo_preprocess(_p(v), C.c_int64(v.size), C.c_float(lower), C.c_float(upper),
                                C.c_double(out_min), C.c_double(out_max), _p(out)))
    return out


def isotropic_grid(grid, mm):
    """register.rs:112-129: the grid resample_isotropic produces."""
    out = Grid()
    _check(lib().fwo_isotropic_grid(C.byref(grid), C.c_double(mm), C.byref(out)))
    return out


def resample_isotropic(grid, img, mm):
    """register.rs:112-146: (grid, image) resampled onto the isotropic mm grid."""
    og = isotropic_grid(grid, mm)
    img = _f64(img)
    out = np.empty(grid_shape(og))
    _check(lib().fwo_resample_isotropic(C.byref(grid), _p(img), C.c_double(mm), _p(out)))
    return og, out


def point_to_index(grid, p):
    out = (C.c_double * 3)()
    _check(lib().fwo_point_to_index(C.byref(grid), (C.c_double * 3)(*p), out))
    return np.array(out[:])


def index_to_point(grid, c):
    out = (C.c_double * 3)()
    _check(lib().fwo_index_to_point(C.byref(grid), (C.c_double * 3)(*c), out))
    return np.array(out[:])


def mt19937(seed, n):
    out = np.empty(n, np.uint32)
    lib().fwo_mt19937(C.c_uint32(seed), C.c_int64(n), _p(out))
    return out


def sample_points_regular(grid, percentage, seed):
    n = lib().fwo_sample_points_regular(C.byref(grid), percentage, seed, None, 0)
    out = np.empty((n, 3), np.float64)
    lib().fwo_sample_points_regular(C.byref(grid), percentage, seed, _p(out), n)
    return out


def mask_inside(mask_grid, mask, points):
    """MaskVolume::is_inside (mask.rs:76-110) for every point (rows of `points`, LPS mm): the
    nearest voxel of the mask on its own grid, rounding half up, inside the buffer and not zero.
    Test infrastructure, in numpy: the grid map is grid.rs:131-156 (point_to_index)."""
    pts = np.asarray(points, np.float64).reshape(-1, 3)
    d = np.array(mask_grid.direction[:]).reshape(3, 3)
    sp = np.array(mask_grid.spacing[:])
    org = np.array(mask_grid.origin[:])
    inv = np.linalg.inv(d * sp[None, :])
    c = (pts - org) @ inv.T
    r = np.floor(c + 0.5)
    size = np.array(mask_grid.size[:])
    ok = np.all((r >= 0) & (r < size), axis=1)
    q = np.where(ok[:, None], r, 0).astype(np.int64)
    m = np.asarray(mask).reshape(size[2], size[1], size[0])
    return ok & (m[q[:, 2], q[:, 1], q[:, 0]] != 0)


def bspline3(u):
    return lib().fwo_bspline3(u)


def bspline3_derivative(u):
    return lib().fwo_bspline3_derivative(u)


def prepare_samples(fgrid, fixed, mgrid, moving, points, bins=32):
    points = _f64(points)
    n = points.shape[0]
    kept = np.empty_like(points)
    fbin = np.empty(n, np.uint32)
    k = C.c_int64()
    b = MiBinning()
    _check(lib().fwo_prepare_samples(C.byref(fgrid), _p(_f64(fixed)), C.byref(mgrid),
                                     _p(_f64(moving)), _p(points), C.c_int64(n), C.c_int32(bins),
                                     _p(kept), _p(fbin), C.byref(k), C.byref(b)))
    return kept[:k.value].copy(), fbin[:k.value].copy(), b


def linear_transform(kind="euler", parameters=None, center=(0, 0, 0), zyx=False,
                     outer_matrix=None, outer_translation=(0, 0, 0), outer_center=(0, 0, 0)):
    t = LinearTransform()
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


def linear_map(t):
    a = Affine()
    lib().fwo_linear_map(C.byref(t), C.byref(a))
    return np.array(a.matrix[:]).reshape(3, 3), np.array(a.offset[:])


def linear_jacobian(t, p):
    cols = np.zeros(36)
    n = lib().fwo_linear_jacobian(C.byref(t), (C.c_double * 3)(*p), _p(cols))
    return cols.reshape(12, 3)[:n].copy()


def mi_evaluate(binning, mgrid, moving, points, fixed_bin, t, want_derivative=True):
    points = _f64(points)
    fixed_bin = np.ascontiguousarray(fixed_bin, np.uint32)
    n = points.shape[0]
    value = C.c_double()
    deriv = np.zeros(12)
    nv = C.c_int64()
    joint = np.zeros(binning.bins * binning.bins)
    _check(lib().fwo_mi_evaluate(C.byref(binning), C.byref(mgrid), _p(_f64(moving)), _p(points),
                                 _p(fixed_bin), C.c_int64(n), C.byref(t),
                                 C.c_int32(int(want_derivative)), C.byref(value), _p(deriv),
                                 C.byref(nv), _p(joint)))
    params = 6 if t.kind == 0 else 12
    return value.value, deriv[:params].copy(), nv.value, joint.reshape(binning.bins, -1)


def convergence_value(values, window, total):
    v = _f64(values)
    return lib().fwo_convergence_value(_p(v), len(v), window, total)


def syn_recipe(gradient_step=0.1, update_variance=3.0, total_variance=0.0, cc_radius=4,
               iterations=(100, 70, 50, 20), shrink=(8, 4, 2, 1), sigmas=(3, 2, 1, 0),
               sigma_units_mm=False, convergence_threshold=1e-6, convergence_window=10,
               weights=(1.0,), metrics=None, mi_bins=32):
    """metrics: one per channel, "cc" or "mattes" (SynMetric; all CC by default)."""
    r = SynRecipe()
    r.gradient_step = gradient_step
    r.update_field_variance = update_variance
    r.total_field_variance = total_variance
    r.cc_radius = cc_radius
    r.levels = len(iterations)
    for k in range(len(iterations)):
        r.iterations[k] = int(iterations[k])
        r.shrink_factors[k] = int(shrink[k])
        r.smoothing_sigmas[k] = float(sigmas[k])
    r.sigma_units_mm = int(bool(sigma_units_mm))
    r.convergence_threshold = convergence_threshold
    r.convergence_window = convergence_window
    r.channels = len(weights)
    for k, w in enumerate(weights):
        r.channel_weights[k] = float(w)
    for k, m in enumerate(metrics or ["cc"] * len(weights)):
        r.channel_metrics[k] = {"cc": 0, "mattes": 1}[m]
    r.mi_bins = int(mi_bins)
    return r


def syn_level_grid(recipe, fixed_grid, level):
    out = Grid()
    _check(lib().fwo_syn_level_grid(C.byref(recipe), C.byref(fixed_grid), C.c_int32(level),
                                    C.byref(out)))
    return out


def _ptrs(arrs):
    return (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


class SynMasks(C.Structure):
    _fields_ = [("fixed_grid", C.POINTER(Grid)), ("fixed", C.POINTER(C.c_double)),
                ("moving_grid", C.POINTER(Grid)), ("moving", C.POINTER(C.c_double))]


def _masks(masks):
    """masks = None or dict(fixed_grid, fixed, moving_grid, moving) (either side may be None).
    Returns (struct or None, arrays kept alive)."""
    if masks is None:
        return None, []
    keep = []
    m = SynMasks()
    for side in ("fixed", "moving"):
        data = masks.get(side)
        if data is not None:
            arr = _f64(data)
            keep.append(arr)
            setattr(m, side, arr.ctypes.data_as(C.POINTER(C.c_double)))
            setattr(m, side + "_grid", C.pointer(masks[side + "_grid"]))
    return m, keep


def syn_step(recipe, level_grid, fixed_grid, fixed_smooth, moving_grid, moving_smooth, initial,
             state, masks=None):
    """One SyN iteration from ``state`` = dict(f2m, f2m_inv, m2m, m2m_inv) (updated in place).
    Returns (record, fixed_update, moving_update)."""
    fs = [_f64(a) for a in fixed_smooth]
    ms = [_f64(a) for a in moving_smooth]
    shape = grid_shape(level_grid) + (3,)
    fu, mu = np.zeros(shape), np.zeros(shape)
    rec = SynIteration()
    for k in ("f2m", "f2m_inv", "m2m", "m2m_inv"):
        state[k] = _f64(state[k])
    cm, _keep = _masks(masks)
    _check(lib().fwo_syn_step_masked(C.byref(recipe), C.byref(level_grid), C.byref(fixed_grid),
                                     _ptrs(fs), C.byref(moving_grid), _ptrs(ms),
                                     None if initial is None else C.byref(initial),
                                     None if cm is None else C.byref(cm),
                                     _p(state["f2m"]), _p(state["f2m_inv"]), _p(state["m2m"]),
                                     _p(state["m2m_inv"]), _p(fu), _p(mu), C.byref(rec)))
    return rec, fu, mu


def syn_run(recipe, fixed_grid, fixed, moving_grid, moving, initial=None, cap=100000,
            masks=None, prior=None):
    """Whole SyN stage; fixed/moving are lists (one image per channel). `prior` = None or
    (grid, warp, inverse_warp): the earlier SyN stages' collapsed fields (run_syn_from)."""
    fs = [_f64(a) for a in fixed]
    ms = [_f64(a) for a in moving]
    last = syn_level_grid(recipe, fixed_grid, recipe.levels - 1)
    shape = grid_shape(last) + (3,)
    warp_out, inv_out = np.zeros(shape), np.zeros(shape)
    recs = (SynIteration * cap)()
    count = C.c_int64()
    cm, _keep = _masks(masks)
    pg, pw, pi = (None, None, None) if prior is None else (prior[0], _f64(prior[1]),
                                                           _f64(prior[2]))
    _check(lib().fwo_syn_run_from(C.byref(recipe), C.byref(fixed_grid), _ptrs(fs),
                                  C.byref(moving_grid), _ptrs(ms),
                                  None if initial is None else C.byref(initial),
                                  None if cm is None else C.byref(cm),
                                  None if pg is None else C.byref(pg), _p(pw), _p(pi),
                                  _p(warp_out), _p(inv_out), recs, C.c_int64(cap),
                                  C.byref(count)))
    return warp_out, inv_out, [recs[i] for i in range(min(count.value, cap))], last


def mi_dense(fgrid, fixed, mgrid, moving, field, bins, fmask_grid=None, fmask=None,
             mmask_grid=None, mmask=None):
    """Dense Mattes MI (value, num_valid, derivative AoS) with the moving point p + field[p]."""
    fixed, moving, field = _f64(fixed), _f64(moving), _f64(field)
    fmask = None if fmask is None else _f64(fmask)
    mmask = None if mmask is None else _f64(mmask)
    value = C.c_double()
    nv = C.c_int64()
    deriv = np.zeros(grid_shape(fgrid) + (3,))
    _check(lib().fwo_mi_dense(C.byref(fgrid), _p(fixed), C.byref(mgrid), _p(moving), _p(field),
                              None if fmask_grid is None else C.byref(fmask_grid), _p(fmask),
                              None if mmask_grid is None else C.byref(mmask_grid), _p(mmask),
                              C.c_int32(bins), C.byref(value), C.byref(nv), _p(deriv)))
    return value.value, nv.value, deriv


# ---- the linear-stage optimiser (optimizer.rs:60-435) -------------------------------------------

class CgSettings(C.Structure):
    _fields_ = [("max_step_mm", C.c_double), ("lower_limit", C.c_double),
                ("upper_limit", C.c_double), ("epsilon", C.c_double),
                ("max_line_search_iterations", C.c_int32), ("iterations", C.c_int32),
                ("convergence_threshold", C.c_double), ("convergence_window", C.c_int32),
                ("small_parameter_variation", C.c_double)]


class CgTrace(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32),
                ("converged_value", C.c_double), ("best_value", C.c_double),
                ("initial_learning_rate", C.c_double), ("final_learning_rate", C.c_double),
                ("line_search_evaluations", C.c_uint64), ("scales", C.c_double * 12),
                ("nvalues", C.c_int64)]


_VALUE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(LinearTransform), C.POINTER(C.c_double))
_VD_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(LinearTransform), C.POINTER(C.c_double),
                     C.POINTER(C.c_double))


def cg_settings_ants(max_step_mm=0.1, iterations=100, threshold=1e-6, window=10):
    """CgSettings::ants (optimizer.rs:94-106)."""
    s = CgSettings()
    s.max_step_mm, s.lower_limit, s.upper_limit, s.epsilon = max_step_mm, 0.0, 2.0, 0.2
    s.max_line_search_iterations, s.iterations = 20, iterations
    s.convergence_threshold, s.convergence_window = threshold, window
    s.small_parameter_variation = 0.01
    return s


def estimate_scales(corners, t, small=0.01):
    n = 6 if t.kind == 0 else 12
    out = (C.c_double * 12)()
    c = (C.c_double * 24)(*np.asarray(corners, np.float64).ravel())
    _check(lib().fwo_estimate_scales(c, C.byref(t), C.c_double(small), out))
    return list(out[:n])


def estimate_step_scale(corners, t, step, small=0.01):
    c = (C.c_double * 24)(*np.asarray(corners, np.float64).ravel())
    s = (C.c_double * 12)(*list(step))
    lib().fwo_estimate_step_scale.restype = C.c_double
    return lib().fwo_estimate_step_scale(c, C.byref(t), s, C.c_double(small))


def cg_optimize_level(value, value_and_derivative, corners, t, settings, cap=100000):
    """optimise_level over Python callables; returns (best transform, trace dict)."""
    n = 6 if t.kind == 0 else 12

    def v_cb(user, tt, out):
        out[0] = float(value(tt.contents))
        return 0

    def vd_cb(user, tt, out, d):
        v, der = value_and_derivative(tt.contents)
        out[0] = float(v)
        for i in range(n):
            d[i] = float(der[i])
        return 0

    c = (C.c_double * 24)(*np.asarray(corners, np.float64).ravel())
    tt = LinearTransform.from_buffer_copy(t)
    tr = CgTrace()
    vals = (C.c_double * cap)()
    f1, f2 = _VALUE_FN(v_cb), _VD_FN(vd_cb)
    _check(lib().fwo_cg_optimize_level(C.byref(settings), c, C.byref(tt), f1, f2, None,
                                       C.byref(tr), vals, C.c_int64(cap)))
    return tt, {"iterations": tr.iterations, "converged": bool(tr.converged),
                "best_value": tr.best_value, "initial_learning_rate": tr.initial_learning_rate,
                "final_learning_rate": tr.final_learning_rate,
                "line_search_evaluations": tr.line_search_evaluations,
                "scales": list(tr.scales[:n]), "values": list(vals[:min(tr.nvalues, cap)])}
