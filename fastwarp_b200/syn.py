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
    # SynMetric per channel (recipe.rs channel_metrics): "cc" or "mattes"; empty = all CC
    channel_metrics: List[str] = field(default_factory=list)
    mi_bins: int = 32

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
        metrics = self.channel_metrics or ["cc"] * r.channels
        if len(metrics) != r.channels:
            raise N.FastwarpError(N.FW_ERR_INVALID, "syn recipe: channel metrics must have one "
                                  "entry per channel weight")
        for k, m in enumerate(metrics):
            if m not in ("cc", "mattes"):
                raise N.FastwarpError(N.FW_ERR_INVALID, f"syn recipe: unknown metric {m!r}")
            r.channel_metrics[k] = 0 if m == "cc" else 1
        r.mi_bins = int(self.mi_bins)
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
            moving_grid: N.Grid, moving: list, initial: N.Affine | None = None,
            fixed_mask=None, moving_mask=None) -> SynResult:
    """run_syn (syn.rs:555-564) from host images (one float array per channel). Masks are
    (grid, array) pairs on any grid (recipe.rs fixed_mask / moving_mask) or None."""
    if fixed_mask is not None or moving_mask is not None:
        fi = [backend.upload_image(fixed_grid, a) for a in fixed]
        mi = [backend.upload_image(moving_grid, a) for a in moving]
        fm = None if fixed_mask is None else backend.upload_image(*fixed_mask)
        mm = None if moving_mask is None else backend.upload_image(*moving_mask)
        w, iw, recs = run_syn_device(backend, recipe, fi, mi, initial, fm, mm)
        last = level_grid(recipe, fixed_grid, recipe.to_c().levels - 1)
        return SynResult(backend.download_field(w).astype(np.float32),
                         backend.download_field(iw).astype(np.float32), last, recs)
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
                   moving: List[Image], initial: N.Affine | None = None,
                   fixed_mask: Image | None = None, moving_mask: Image | None = None,
                   prior: tuple | None = None):
    """The same on device-resident images; returns (warp Field, inverse Field, records).
    `prior` = (warp Field, inverse Field) of earlier SyN stages makes this run_syn_from
    (syn.rs:620-660): a later stage, collapsed with the prior."""
    r = recipe.to_c()
    fp = (C.c_void_p * len(fixed))(*[im.handle.value for im in fixed])
    mp = (C.c_void_p * len(moving))(*[im.handle.value for im in moving])
    cap = max(1, sum(recipe.iterations))
    recs = (N.SynIteration * cap)()
    count = C.c_int64()
    w, iw = C.c_void_p(), C.c_void_p()
    fm = None if fixed_mask is None else fixed_mask.handle
    mm = None if moving_mask is None else moving_mask.handle
    init = None if initial is None else C.byref(initial)
    if prior is None:
        check(lib().fw_syn_run_device_masked(backend.ctx, C.byref(r), fp, mp, fm, mm, init,
                                             C.byref(w), C.byref(iw), recs, C.c_int64(cap),
                                             C.byref(count)))
    else:
        check(lib().fw_syn_run_device_from(backend.ctx, C.byref(r), fp, mp, fm, mm, init,
                                           prior[0].handle, prior[1].handle, C.byref(w),
                                           C.byref(iw), recs, C.c_int64(cap), C.byref(count)))
    return Field(backend, w), Field(backend, iw), _records(recs, min(count.value, cap))


def run_syn_from(backend: CudaBackend, recipe: SynRecipe, fixed_grid: N.Grid, fixed: list,
                 moving_grid: N.Grid, moving: list, initial: N.Affine | None,
                 prior_warp, prior_inverse_warp, fixed_mask=None,
                 moving_mask=None) -> SynResult:
    """run_syn_from (syn.rs:620-660) from host images: a later SyN stage whose moving side goes
    through the earlier stages' collapsed fields (AoS arrays on the grid of this stage's last
    level, as SynResult.warp / inverse_warp hold them); the result is collapsed with them."""
    last = level_grid(recipe, fixed_grid, recipe.to_c().levels - 1)
    fi = [backend.upload_image(fixed_grid, a) for a in fixed]
    mi = [backend.upload_image(moving_grid, a) for a in moving]
    fm = None if fixed_mask is None else backend.upload_image(*fixed_mask)
    mm = None if moving_mask is None else backend.upload_image(*moving_mask)
    prior = (backend.upload_field(last, prior_warp), backend.upload_field(last, prior_inverse_warp))
    w, iw, recs = run_syn_device(backend, recipe, fi, mi, initial, fm, mm, prior)
    return SynResult(backend.download_field(w).astype(np.float32),
                     backend.download_field(iw).astype(np.float32), last, recs)


class WindowConvergenceMonitor:
    """ITK's window convergence monitor (convergence.rs:47-126), on the host."""

    def __init__(self, window: int):
        self.window = window
        self.values = []
        self.total = 0.0

    def add(self, v: float):
        self.values.append(v)
        if len(self.values) > self.window:
            self.values.pop(0)
        self.total += abs(v)

    def value(self) -> float:
        if len(self.values) < self.window:
            return float(np.finfo(np.float64).max)
        if self.window < 2:
            return 0.0
        r = 1.0 / ((11.0 - 1.0) * 0.1)
        eps = r * 0.1 * 1e-3
        delta, omega = [0.0, 0.0], [0.0, 0.0]
        for n, e in enumerate(self.values):
            p = (n / (self.window - 1)) * r
            if abs(p - 1.0) <= eps:
                p = 1.0 - eps
            if p < 0.0 and abs(p) <= eps:
                p = 0.0
            t = p - np.floor(p)
            w = (1.0 - t, t)
            w2 = w[0] * w[0] + w[1] * w[1]
            v = e / self.total
            for j in range(2):
                omega[j] += w[j] * w[j]
                delta[j] += v * (w[j] ** 3 / w2)
        phi = [0.0, 0.0]
        for j in range(2):
            if abs(omega[j]) > np.finfo(np.float64).eps:
                q = delta[j] / omega[j]
                phi[j] = q if np.isfinite(q) else 0.0
        return phi[0] - phi[1]


def run_syn_ops(backend: CudaBackend, recipe: SynRecipe, fixed_grid: N.Grid, fixed: list,
                moving_grid: N.Grid, moving: list, initial: N.Affine | None = None):
    """syn_fields (syn.rs:776-986) driven op by op through the Backend operations, every op a
    synchronous call -- how the reference's loop drives an engine. Returns (warp, inverse_warp,
    records) with the fields as host AoS float64 on the last level grid."""
    from .backend import shrink_factors, shrink_grid
    b = backend
    C_ = len(recipe.channel_weights)
    wsum = sum(recipe.channel_weights)
    wn = [w / wsum for w in recipe.channel_weights]
    fi = [b.upload_image(fixed_grid, np.ascontiguousarray(a, np.float32)) for a in fixed]
    mi = [b.upload_image(moving_grid, np.ascontiguousarray(a, np.float32)) for a in moving]
    F = Fi = M = Mi = None
    records = []
    eps = np.finfo(np.float64).eps
    for level, limit in enumerate(recipe.iterations):
        grid = shrink_grid(fixed_grid, shrink_factors(recipe.shrink_factors[level],
                                                      tuple(fixed_grid.spacing)))
        sigma = recipe.smoothing_sigmas[level]
        if sigma > 0:
            def sig(g):
                return [sigma if recipe.sigma_units_mm else sigma * g.spacing[a] for a in range(3)]
            fs = [b.smooth_recursive(im, sig(fixed_grid)) for im in fi]
            ms = [b.smooth_recursive(im, sig(moving_grid)) for im in mi]
        else:
            fs, ms = fi, mi
        if F is None:
            F, Fi, M, Mi = (b.zero_field(grid) for _ in range(4))
        else:
            F, Fi, M, Mi = (b.resample_field(x, grid) for x in (F, Fi, M, Mi))
        monitor = WindowConvergenceMonitor(recipe.convergence_window)
        current, converged = 0, False
        while current < limit and not converged:
            current += 1
            fmid = [b.warp_through_field(fs[c], Fi) for c in range(C_)]
            mmid = [b.warp_through_field(ms[c], Mi, None, initial) for c in range(C_)]
            sides = []
            for side in range(2):
                sides.append({"values": [], "grad": None, "mag": 0.0})
            metrics = recipe.channel_metrics or ["cc"] * C_
            for c in range(C_):
                # syn.rs:350-398: the channel's metric pair, with norms for several channels
                if metrics[c] == "mattes":
                    pair, norms = b.mi_value_derivative_pair_with_norms(fmid[c], mmid[c],
                                                                        recipe.mi_bins)
                else:
                    pair, norms = b.cc_value_derivative_pair_with_norms(fmid[c], mmid[c],
                                                                        recipe.cc_radius)
                (vf, df), (vm, dm) = pair
                if C_ == 1:
                    sides[0]["values"].append(vf)
                    sides[1]["values"].append(vm)
                    sides[0]["grad"], sides[1]["grad"] = df, dm
                else:
                    for side, (v, d, nrm) in enumerate([(vf, df, norms[0]), (vm, dm, norms[1])]):
                        s = sides[side]
                        s["values"].append(v)
                        if s["grad"] is None:
                            s["grad"] = b.zero_field(grid)
                        if not np.isfinite(nrm):
                            raise N.FastwarpError(N.FW_ERR_NOT_FINITE,
                                                  "syn: the metric gradient is not finite")
                        s["mag"] += nrm
                        if nrm > eps:
                            b.axpy(s["grad"], wn[c] / nrm, d)
            for s in sides:
                if C_ > 1:
                    b.scale(s["grad"], s["mag"] / C_)
                s["grad"] = b.smooth_field(s["grad"], recipe.update_field_variance)
            mF, mM = b.max_scaled_norm_pair(sides[0]["grad"], sides[1]["grad"])
            if not (np.isfinite(mF) and np.isfinite(mM)):
                raise N.FastwarpError(N.FW_ERR_NOT_FINITE, "syn: the metric gradient is not finite")
            scales = []
            for s, mx in zip(sides, (mF, mM)):
                sc = recipe.gradient_step / mx if mx > 0.0 else recipe.gradient_step
                b.scale(s["grad"], sc)
                scales.append(sc)
            stats = []
            for side, (field, inverse) in enumerate([(F, Fi), (M, Mi)]):
                composed = b.compose(sides[side]["grad"], field)
                tmp = b.smooth_field(composed, recipe.total_field_variance)
                (new_inv, s1), (new_field, s2) = b.invert_pair(tmp, inverse)
                stats += [s1, s2]
                if side == 0:
                    F, Fi = new_field, new_inv
                else:
                    M, Mi = new_field, new_inv
            energy = 0.5 * (sides[0]["values"][0] + sides[1]["values"][0])
            monitor.add(energy)
            cv = monitor.value()
            converged = cv < recipe.convergence_threshold
            records.append({"level": level, "energy": energy, "convergence_value": cv,
                            "fixed_update_scale": scales[0], "moving_update_scale": scales[1],
                            "inversions": stats})
    warp = b.download_field(b.compose(Mi, F))
    inverse = b.download_field(b.compose(Fi, M))
    return warp, inverse, records


def syn_step(backend: CudaBackend, recipe: SynRecipe, fixed: List[Image], moving: List[Image],
             initial: N.Affine | None, state: dict, want_updates: bool = True,
             fixed_mask: Image | None = None, moving_mask: Image | None = None):
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
    check(lib().fw_syn_step_masked(backend.ctx, C.byref(r), fp, mp,
                            None if fixed_mask is None else fixed_mask.handle,
                            None if moving_mask is None else moving_mask.handle,
                            None if initial is None else C.byref(initial),
                            state["f2m"].handle, state["f2m_inv"].handle, state["m2m"].handle,
                            state["m2m_inv"].handle,
                            None if fu is None else fu.ctypes.data_as(C.c_void_p),
                            None if mu is None else mu.ctypes.data_as(C.c_void_p),
                            C.byref(rec)))
    return _records([rec], 1)[0], fu, mu


@dataclass
class BatchResult:
    """The batching form's outcome: per subject its SynResult (None when it failed) and status,
    and the autotuner's per-level choices with each level's device time."""
    subjects: list
    statuses: list
    tuning: list
    level_ms: list
    device_bytes: int
    prepare_ms: list = None
    finish_ms: float = 0.0


def run_syn_batch(backend: CudaBackend, recipe: SynRecipe, fixed: List[Image],
                  subjects: list, download: bool = True) -> BatchResult:
    """fw_batch_syn_run: every subject registered to the one template `fixed` (device images, one
    per channel) in lockstep; `subjects` is a list of (moving: [Image per channel], initial
    affine or None). Each subject's fields are downloaded (AoS float32) unless download is False,
    when the SynResult holds the device Fields instead."""
    r = recipe.to_c()
    B = len(subjects)
    subj = (N.BatchSubject * B)()
    for b, (moving, initial) in enumerate(subjects):
        for c, im in enumerate(moving):
            subj[b].moving[c] = im.handle
        if initial is not None:
            subj[b].initial = initial
            subj[b].has_initial = 1
    fp = (C.c_void_p * len(fixed))(*[im.handle for im in fixed])
    warps = (C.c_void_p * B)()
    invs = (C.c_void_p * B)()
    cap = max(1, sum(recipe.iterations))
    recs = (N.SynIteration * (cap * B))()
    counts = (C.c_int64 * B)()
    statuses = (C.c_int32 * B)()
    rep = N.BatchReport()
    check(lib().fw_batch_syn_run(backend.ctx, C.byref(r), fp, C.c_int32(B), subj, warps, invs,
                                 recs, C.c_int64(cap), counts, statuses, C.byref(rep)))
    last = level_grid(recipe, fixed[0].grid, r.levels - 1)
    out = []
    for b in range(B):
        if statuses[b] != 0:
            out.append(None)
            continue
        w, iw = Field(backend, C.c_void_p(warps[b])), Field(backend, C.c_void_p(invs[b]))
        its = _records(recs[b * cap:(b + 1) * cap], counts[b])
        if download:
            out.append(SynResult(backend.download_field(w).astype(np.float32),
                                 backend.download_field(iw).astype(np.float32), last, its))
            w.free()
            iw.free()
        else:
            out.append(SynResult(w, iw, last, its))
    tuning = []
    for lv in range(r.levels):
        t = rep.tuning[lv]
        tuning.append({k: (list(getattr(t, k)) if k in ("grid_size", "kernel_ms") else getattr(t, k))
                       for k, _ in N.BatchTuning._fields_})
    return BatchResult(out, list(statuses), tuning, list(rep.level_ms[:r.levels]),
                       int(rep.device_bytes), list(rep.prepare_ms[:r.levels]),
                       float(rep.finish_ms))
