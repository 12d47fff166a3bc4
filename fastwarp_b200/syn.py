"""The SyN stage (syn.rs:555-753 `run_syn`) on the device, and the cohort recipes (recipe.rs)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List

import numpy as np

from . import _native as N
from ._native import check, lib
from .backend import CudaBackend, Field, Image, grid_shape


@dataclass
class SynRecipe:
    """SynRecipe (recipe.rs:52-100). Variances are in squared voxels of the level grid."""
    gradient_step: float = 0.1
    update_field_variance: float = 3.0
    total_field_variance: float = 0.0
    cc_radius: int = 4
    iterations: List[int] = field(default_factory=lambda: [100, 70, 50, 20])
    shrink_factors: List[int] = field(default_factory=lambda: [8, 4, 2, 1])
    smoothing_sigmas: List[float] = field(default_factory=lambda: [3.0, 2.0, 1.0, 0.0])
    sigma_units_mm: bool = False
    convergence_threshold: float = 1e-6
    convergence_window: int = 10
    channel_weights: List[float] = field(default_factory=lambda: [1.0])

    @staticmethod
    def cohort() -> "SynRecipe":
        """SyN[0.1,3,0], CC[...,1,4], [100x70x50x20,1e-6,10], 8x4x2x1, 3x2x1x0vox."""
        return SynRecipe()

    @staticmethod
    def cohort_channels(channels: int) -> "SynRecipe":
        n = max(channels, 1)
        return SynRecipe(channel_weights=[1.0 / n] * n)

    def to_c(self) -> N.SynRecipe:
        r = N.SynRecipe()
        r.gradient_step = self.gradient_step
        r.update_field_variance = self.update_field_variance
        r.total_field_variance = self.total_field_variance
        r.cc_radius = self.cc_radius
        r.levels = len(self.iterations)
        if not (len(self.shrink_factors) == len(self.smoothing_sigmas) == r.levels):
            raise N.FastwarpError(N.FW_ERR_INVALID, "syn recipe: iterations, shrink factors and "
                                  "smoothing sigmas must have one entry per level")
        if r.levels > N.MAX_LEVELS or len(self.channel_weights) > N.MAX_CHANNELS:
            raise N.FastwarpError(N.FW_ERR_INVALID, "syn recipe: too many levels or channels")
        for k in range(r.levels):
            r.iterations[k] = int(self.iterations[k])
            r.shrink_factors[k] = int(self.shrink_factors[k])
            r.smoothing_sigmas[k] = float(self.smoothing_sigmas[k])
        r.sigma_units_mm = int(bool(self.sigma_units_mm))
        r.convergence_threshold = self.convergence_threshold
        r.convergence_window = self.convergence_window
        r.channels = len(self.channel_weights)
        for k, w in enumerate(self.channel_weights):
            r.channel_weights[k] = float(w)
        return r


@dataclass
class SynResult:
    """SynResult (syn.rs:130-145): the two fields on the last level grid (AoS float32, LPS mm)
    and the per-iteration records."""
    warp: np.ndarray
    inverse_warp: np.ndarray
    grid: N.Grid
    iterations: list


def level_grid(recipe: SynRecipe, fixed_grid: N.Grid, level: int) -> N.Grid:
    out = N.Grid()
    r = recipe.to_c()
    check(lib().fw_syn_level_grid(C.byref(r), C.byref(fixed_grid), C.c_int32(level),
                                  C.byref(out)))
    return out


def _records(recs, n):
    out = []
    for i in range(n):
        r = recs[i]
        out.append({
            "level": r.level, "energy": r.energy, "energy_weighted": r.energy_weighted,
            "convergence_value": r.convergence_value,
            "fixed_update_scale": r.fixed_update_scale,
            "moving_update_scale": r.moving_update_scale,
            "inversions": [(s.iterations, s.mean_error_norm, s.max_error_norm)
                           for s in r.inversions],
        })
    return out


def run_syn(backend: CudaBackend, recipe: SynRecipe, fixed_grid: N.Grid, fixed: list,
            moving_grid: N.Grid, moving: list, initial: N.Affine | None = None) -> SynResult:
    """run_syn (syn.rs:555-564) from host images (one float array per channel)."""
    r = recipe.to_c()
    fs = [np.ascontiguousarray(a, np.float32) for a in fixed]
    ms = [np.ascontiguousarray(a, np.float32) for a in moving]
    last = level_grid(recipe, fixed_grid, r.levels - 1)
    shape = grid_shape(last) + (3,)
    warp = np.empty(shape, np.float32)
    inv = np.empty(shape, np.float32)
    cap = max(1, sum(recipe.iterations))
    recs = (N.SynIteration * cap)()
    count = C.c_int64()
    fp = (C.c_void_p * len(fs))(*[a.ctypes.data for a in fs])
    mp = (C.c_void_p * len(ms))(*[a.ctypes.data for a in ms])
    check(lib().fw_syn_run(backend.ctx, C.byref(r), C.byref(fixed_grid), fp,
                           C.byref(moving_grid), mp,
                           None if initial is None else C.byref(initial),
                           warp.ctypes.data_as(C.c_void_p), inv.ctypes.data_as(C.c_void_p),
                           recs, C.c_int64(cap), C.byref(count)))
    return SynResult(warp, inv, last, _records(recs, min(count.value, cap)))


def run_syn_device(backend: CudaBackend, recipe: SynRecipe, fixed: List[Image],
                   moving: List[Image], initial: N.Affine | None = None):
    """The same on device-resident images; returns (warp Field, inverse Field, records)."""
    r = recipe.to_c()
    fp = (C.c_void_p * len(fixed))(*[im.handle.value for im in fixed])
    mp = (C.c_void_p * len(moving))(*[im.handle.value for im in moving])
    cap = max(1, sum(recipe.iterations))
    recs = (N.SynIteration * cap)()
    count = C.c_int64()
    w, iw = C.c_void_p(), C.c_void_p()
    check(lib().fw_syn_run_device(backend.ctx, C.byref(r), fp, mp,
                                  None if initial is None else C.byref(initial),
                                  C.byref(w), C.byref(iw), recs, C.c_int64(cap),
                                  C.byref(count)))
    return Field(backend, w), Field(backend, iw), _records(recs, min(count.value, cap))


def syn_step(backend: CudaBackend, recipe: SynRecipe, fixed: List[Image], moving: List[Image],
             initial: N.Affine | None, state: dict, want_updates: bool = True):
    """One SyN iteration (syn.rs:890-958) on device-resident state fields f2m, f2m_inv, m2m,
    m2m_inv (updated in place). Returns (record, fixed_update, moving_update)."""
    r = recipe.to_c()
    fp = (C.c_void_p * len(fixed))(*[im.handle.value for im in fixed])
    mp = (C.c_void_p * len(moving))(*[im.handle.value for im in moving])
    g = state["f2m"].grid
    shape = grid_shape(g) + (3,)
    fu = np.zeros(shape) if want_updates else None
    mu = np.zeros(shape) if want_updates else None
    rec = N.SynIteration()
    check(lib().fw_syn_step(backend.ctx, C.byref(r), fp, mp,
                            None if initial is None else C.byref(initial),
                            state["f2m"].handle, state["f2m_inv"].handle, state["m2m"].handle,
                            state["m2m_inv"].handle,
                            None if fu is None else fu.ctypes.data_as(C.c_void_p),
                            None if mu is None else mu.ctypes.data_as(C.c_void_p),
                            C.byref(rec)))
    return _records([rec], 1)[0], fu, mu
