"""The continuous-batching registration server (include/fastwarp_serve.h) from Python.

A `Server` owns N execution slots on one GPU (each a context with its own stream). Requests are
queued at once and admitted as slots free up and their device-memory estimate fits the HBM
budget; admitted registrations run concurrently and their kernels overlap on the device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from ._native import check, lib
from .backend import Field, Image, grid_shape
from .syn import SynRecipe


class SynRequest(C.Structure):
    _fields_ = [("recipe", N.SynRecipe), ("fixed_grid", N.Grid), ("moving_grid", N.Grid),
                ("fixed", C.c_void_p), ("moving", C.c_void_p), ("fixed_dev", C.c_void_p),
                ("moving_dev", C.c_void_p), ("initial", N.Affine), ("has_initial", C.c_int32),
                ("keep_on_device", C.c_int32), ("tag", C.c_uint64),
                ("fixed_mask_grid", N.Grid), ("moving_mask_grid", N.Grid),
                ("fixed_mask", C.c_void_p), ("moving_mask", C.c_void_p),
                ("fixed_mask_dev", C.c_void_p), ("moving_mask_dev", C.c_void_p)]


class _ResultBuffers:
    """Owns the host buffers of one server result (fw_server_result_free when collected)."""

    def __init__(self, result):
        self.result = result

    def array(self, address, shape):
        n = int(np.prod(shape))
        buf = (C.c_float * n).from_address(address)
        buf._owner = self  # numpy's view keeps `buf`, `buf` keeps the owner
        return np.ctypeslib.as_array(buf).reshape(shape)

    def __del__(self):
        try:
            lib().fw_server_result_free(C.byref(self.result))
        except Exception:
            pass


class SynResultC(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("status", C.c_int32), ("error", C.c_char * 256),
                ("grid", N.Grid), ("warp", C.c_void_p), ("inverse_warp", C.c_void_p),
                ("warp_dev", C.c_void_p), ("inverse_dev", C.c_void_p),
                ("iterations", C.c_int64), ("final_energy", C.c_double),
                ("device_bytes", C.c_uint64), ("queued_s", C.c_double), ("run_s", C.c_double),
                ("device_start_ms", C.c_double), ("device_end_ms", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in (
        "submitted", "completed", "failed", "active", "queued", "reserved_bytes",
        "peak_reserved_bytes", "budget_bytes", "kernel_launches", "graph_launches")]


class LinearRequest(C.Structure):
    _fields_ = [("recipe", N.LinearRecipe), ("fixed_grid", N.Grid), ("moving_grid", N.Grid),
                ("fixed", C.c_void_p), ("moving", C.c_void_p), ("fixed_dev", C.c_void_p),
                ("moving_dev", C.c_void_p), ("start", N.LinearTransform), ("tag", C.c_uint64)]


class LinearResultC(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("status", C.c_int32), ("error", C.c_char * 256),
                ("transform", N.LinearTransform), ("nlevels", C.c_int32),
                ("levels", N.LinearLevelTrace * 8), ("device_bytes", C.c_uint64),
                ("queued_s", C.c_double), ("run_s", C.c_double)]


class Server:
    def __init__(self, device: int = 0, budget_bytes: int = 0, slots: int = 4):
        h = C.c_void_p()
        check(lib().fw_server_create(int(device), C.c_uint64(int(budget_bytes)), C.c_int32(slots),
                                     C.byref(h)))
        self.handle = h
        self._keep = {}

    def close(self):
        if self.handle:
            lib().fw_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _request(self, recipe: SynRecipe, fixed_grid, fixed, moving_grid, moving, initial, tag,
                 keep_on_device, fixed_mask=None, moving_mask=None):
        q = SynRequest()
        q.recipe = recipe.to_c()
        q.fixed_grid = fixed_grid
        q.moving_grid = moving_grid
        keep = []
        if isinstance(fixed[0], Image):
            fp = (C.c_void_p * len(fixed))(*[im.handle.value for im in fixed])
            mp = (C.c_void_p * len(moving))(*[im.handle.value for im in moving])
            q.fixed_dev = C.cast(fp, C.c_void_p)
            q.moving_dev = C.cast(mp, C.c_void_p)
            keep = [fp, mp, fixed, moving]
        else:
            fs = [np.ascontiguousarray(a, np.float32) for a in fixed]
            ms = [np.ascontiguousarray(a, np.float32) for a in moving]
            fp = (C.c_void_p * len(fs))(*[a.ctypes.data for a in fs])
            mp = (C.c_void_p * len(ms))(*[a.ctypes.data for a in ms])
            q.fixed = C.cast(fp, C.c_void_p)
            q.moving = C.cast(mp, C.c_void_p)
            keep = [fp, mp, fs, ms]
        if initial is not None:
            q.initial = initial
            q.has_initial = 1
        q.keep_on_device = int(bool(keep_on_device))
        q.tag = int(tag)
        # masks: a device Image, or (grid, host array) copied at submit
        for name, m in (("fixed", fixed_mask), ("moving", moving_mask)):
            if m is None:
                continue
            if isinstance(m, Image):
                setattr(q, name + "_mask_grid", m.grid)
                setattr(q, name + "_mask_dev", m.handle.value)
                keep.append(m)
            else:
                grid, data = m
                arr = np.ascontiguousarray(data, np.float32)
                setattr(q, name + "_mask_grid", grid)
                setattr(q, name + "_mask", arr.ctypes.data)
                keep.append(arr)
        return q, keep

    def estimate(self, recipe, fixed_grid, fixed, moving_grid, moving, initial=None) -> int:
        q, _ = self._request(recipe, fixed_grid, fixed, moving_grid, moving, initial, 0, False)
        b = C.c_uint64()
        check(lib().fw_server_estimate(C.byref(q), C.byref(b)))
        return int(b.value)

    def submit(self, recipe: SynRecipe, fixed_grid, fixed, moving_grid, moving, initial=None,
               tag=0, keep_on_device=False, fixed_mask=None, moving_mask=None) -> int:
        """Queues one SyN registration; `fixed`/`moving` are lists (one per channel) of host
        float arrays or of device `Image`s; masks are a device `Image` or (grid, host array).
        Returns the ticket."""
        q, keep = self._request(recipe, fixed_grid, fixed, moving_grid, moving, initial, tag,
                                keep_on_device, fixed_mask, moving_mask)
        t = C.c_uint64()
        check(lib().fw_server_submit(self.handle, C.byref(q), C.byref(t)))
        self._keep[int(t.value)] = keep  # device images must outlive the request
        return int(t.value)

    def wait(self, ticket: int, timeout: float = -1.0) -> dict:
        r = SynResultC()
        check(lib().fw_server_wait(self.handle, C.c_uint64(ticket), C.c_double(timeout),
                                   C.byref(r)))
        self._keep.pop(ticket, None)
        out = {"tag": r.tag, "status": r.status, "error": r.error.decode(errors="replace"),
               "iterations": r.iterations, "final_energy": r.final_energy,
               "device_bytes": r.device_bytes, "queued_s": r.queued_s, "run_s": r.run_s,
               "latency_s": r.queued_s + r.run_s, "device_start_ms": r.device_start_ms,
               "device_end_ms": r.device_end_ms, "grid": r.grid}
        out["warp_dev"], out["inverse_dev"] = r.warp_dev, r.inverse_dev
        if r.status == 0 and r.warp:
            # the arrays view the result's pinned buffers; they go back to the library's pool
            # when the last array referring to them is gone
            shape = grid_shape(r.grid) + (3,)
            owner = _ResultBuffers(r)
            out["warp"] = owner.array(r.warp, shape)
            out["inverse_warp"] = owner.array(r.inverse_warp, shape)
        else:
            lib().fw_server_result_free(C.byref(r))
        return out

    def submit_linear(self, recipe: N.LinearRecipe, fixed_grid, fixed, moving_grid, moving,
                      start: N.LinearTransform, tag=0) -> int:
        """Queues one linear stage (run_linear_stage); `fixed`/`moving` are host float arrays
        (copied at submit) or device `Image`s. Returns the ticket."""
        q = LinearRequest()
        q.recipe, q.fixed_grid, q.moving_grid, q.start, q.tag = (recipe, fixed_grid, moving_grid,
                                                                 start, int(tag))
        if isinstance(fixed, Image):
            q.fixed_dev, q.moving_dev = fixed.handle.value, moving.handle.value
            keep = [fixed, moving]
        else:
            fa = np.ascontiguousarray(fixed, np.float32)
            ma = np.ascontiguousarray(moving, np.float32)
            q.fixed, q.moving = fa.ctypes.data, ma.ctypes.data
            keep = [fa, ma]
        t = C.c_uint64()
        check(lib().fw_server_submit_linear(self.handle, C.byref(q), C.byref(t)))
        self._keep[int(t.value)] = keep
        return int(t.value)

    def wait_linear(self, ticket: int, timeout: float = -1.0) -> dict:
        r = LinearResultC()
        check(lib().fw_server_wait_linear(self.handle, C.c_uint64(ticket), C.c_double(timeout),
                                          C.byref(r)))
        self._keep.pop(ticket, None)
        n = 6 if r.transform.kind == 0 else 12
        return {"tag": r.tag, "status": r.status, "error": r.error.decode(errors="replace"),
                "transform": r.transform, "parameters": list(r.transform.parameters[:n]),
                "levels": [dict(samples=lv.samples, skipped=bool(lv.skipped),
                                iterations=lv.cg.iterations, best_value=lv.cg.best_value)
                           for lv in r.levels[:r.nlevels]],
                "device_bytes": r.device_bytes, "queued_s": r.queued_s, "run_s": r.run_s}

    @staticmethod
    def free_device_fields(result: dict):
        for k in ("warp_dev", "inverse_dev"):
            if result.get(k):
                lib().fw_field_free(C.c_void_p(result[k]))
                result[k] = None

    def cancel(self, ticket: int) -> None:
        """fw_server_cancel: a queued request ends without running, a running one after the
        iteration in flight; its result then fails with FW_ERR_CANCELLED."""
        check(lib().fw_server_cancel(self.handle, C.c_uint64(ticket)))

    def mark(self):
        check(lib().fw_server_mark(self.handle))

    def stats(self) -> dict:
        s = ServerStats()
        check(lib().fw_server_stats_get(self.handle, C.byref(s)))
        return {k: int(getattr(s, k)) for k, _ in ServerStats._fields_}
