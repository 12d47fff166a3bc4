#!/usr/bin/env python
"""Benchmark: SyN registrations/hour of the config-2 workload on B200.

Workload ("head-1mm"): the SyN stage of the brain-template-shape pipeline, a seeded
193 x 229 x 193 float32 phantom pair at 1 mm (nested ellipsoids 0.2/0.5/0.8, +-20 % bias,
Rician-like noise 0.02; moving = rigid + affine + smooth field of the fixed image), CC radius 4,
shrink 4/2/1, smoothing sigma 2/1/0 voxels, iterations 70/50/20 all run (convergence threshold
-1, so both engines run the same 140 iterations: the recipe the full-size parity test checks
against the oracle), gradient step 0.1, update variance 3, total variance 0. The linear part of
the phantom's map is the SyN stage's initial transform (a converged linear stage).

A second leg times the affine stage's sampled Mattes MI at the same finest level (25 % regular
sampling, 32 bins: S = 2.13 M samples): each pass by CUDA events with its roofline, one value and
one value-and-derivative through the host API, the oracle's evaluation on the host cores beside
them, and the whole linear chain (centre of mass, rigid, affine at shrink 4/2/1, sigma 2/1/0,
500/250/100 iterations, 1e-6 over 10).

One step = one batch of `--concurrency` registrations served together (continuous batching: each
registration on its own stream, admitted as slots free up; `--mode sequential` runs them one at a
time). `value` is registrations/hour with the images resident in HBM, timed with CUDA events on the
engines' streams between barriers, max over ranks; `e2e` is the same through the public host API
(`run_syn`: pinned host images in, AoS float32 fields out, copies inside the timed region).
Every working set here (fields of 100 MB, images of 34 MB per registration) exceeds the 126 MB L2
many times over, so no L2 flush is needed between steps.

`--impl reference` times the reference's CPU engine restated as the f64 oracle (the Rust
reference cannot be built here) on all host cores, on a bounded sample: a few consecutive SyN
iterations per level plus the level smoothing, each step's `ms_per_step` the sample's own wall
time and its value the registrations/hour of the measured per-iteration times times the 70/50/20
iterations both engines run. `--impl reference --full-cpu` times one whole oracle registration
instead (about a minute and a half), which validates that extrapolation.
"""
import argparse
import faulthandler
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
faulthandler.enable()


def log(msg):
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)

ITERATIONS = [70, 50, 20]
SHRINK = [4, 2, 1]
SIGMAS = [2.0, 1.0, 0.0]
SHAPE = (193, 229, 193)
METRIC = "SyN registrations/hour (served vs sequential, same CC); p50/p99 latency"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--mode", choices=["served", "sequential"], default="served")
    p.add_argument("--concurrency", type=int, default=4)
    p.add_argument("--shape", type=str, default=None, help="override nx,ny,nz (tests)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--kernels-only", action="store_true",
                   help="time the kernels of one finest-level iteration only (profiling target)")
    p.add_argument("--reps", type=int, default=20)
    p.add_argument("--no-mi", action="store_true", help="skip the sampled Mattes MI leg")
    p.add_argument("--no-batch", action="store_true", help="skip the batching-form leg")
    p.add_argument("--only", choices=["batch", "mi", "stream"], default=None,
                   help="run one leg alone (profiling target): the batching form or the sampled "
                        "Mattes MI with the linear chain")
    p.add_argument("--subjects", type=int, default=48, help="subjects of the batching leg")
    p.add_argument("--no-chain", action="store_true", help="MI leg without the linear chain")
    p.add_argument("--full-cpu", action="store_true",
                   help="with --impl reference: time one whole oracle registration")
    return p.parse_args()


def time_kernels(b, fimg, mimg, reps):
    """Per-kernel mean ms and algorithmic bytes at the grid of the images (CUDA events on the
    engine's stream)."""
    import ctypes as C

    from fastwarp_b200 import _native as N
    ms = (C.c_double * 7)()
    by = (C.c_double * 7)()
    N.check(N.lib().fw_time_kernels(b.ctx, fimg.handle, mimg.handle, C.c_int32(4),
                                    C.c_double(3.0), C.c_int32(reps), ms, by))
    names = ["warp", "cc_pair", "smooth", "compose", "inv_body", "inv_bound", "inv_fix"]
    t = {k: (ms[i], by[i]) for i, k in enumerate(names)}
    # the body's step kernel alone: the body (bound, step, fix back to back on the stream) less
    # the bound and the fix timed on their own; its bytes are the body's (psi in, field gathered,
    # psi out)
    t["inv_step"] = (max(ms[4] - ms[5] - ms[6], 1e-6), by[4])
    return t


def run_kernels_only(args, local):
    from fastwarp_b200 import CudaBackend
    from fastwarp_b200.phantoms import head_phantom
    shape = tuple(int(x) for x in args.shape.split(",")) if args.shape else SHAPE
    from fastwarp_b200 import make_grid
    g = make_grid(shape)
    fixed = head_phantom(shape)
    moving = head_phantom(shape, seed=7)
    with CudaBackend(local) as b:
        t = time_kernels(b, b.upload_image(g, fixed), b.upload_image(g, moving), args.reps)
    return {"kernels": {k: {"ms": round(v[0], 4), "gbs": round(v[1] / (v[0] / 1000) / 1e9, 1)}
                        for k, v in t.items()}, "shape": shape}


def run_one_leg(args, rank, world, local):
    from fastwarp_b200 import CudaBackend
    b = CudaBackend(local)
    if args.only == "batch":
        out = {"batched": batch_leg(b, rank, args.subjects)}
    elif args.only == "stream":
        out = {"stream": stream_leg(b, rank)}
    else:
        from fastwarp_b200.phantoms import head_pair
        g, fixed, mg, moving, initial = head_pair(SHAPE, seed=20_260_910 + 2 + rank)
        fi, mi = b.upload_image(g, fixed), b.upload_image(mg, moving)
        out = {"mattes_mi": mi_leg(b, g, fixed, mg, moving, initial, fi, mi, rank, world,
                                   chain=not args.no_chain)}
    b.close()
    return out


def recipe():
    from fastwarp_b200 import SynRecipe
    return SynRecipe(gradient_step=0.1, update_field_variance=3.0, total_field_variance=0.0,
                     cc_radius=4, iterations=list(ITERATIONS), shrink_factors=list(SHRINK),
                     smoothing_sigmas=list(SIGMAS), convergence_threshold=-1.0,
                     convergence_window=10, channel_weights=[1.0])


def dist_init(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        import torch
        torch.cuda.set_device(local)
        # only the max-over-ranks time and the summed counts cross ranks (replicas, no data path)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world):
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


class Clocks:
    """nvidia-smi samples during the timed region (SM clocks and throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def kernel_traffic():
    """dram bytes per voxel of each kernel from the committed ncu summary (or None)."""
    path = os.path.join(ROOT, "profiles", "kernel_traffic.json")
    try:
        return json.load(open(path))
    except (OSError, ValueError):
        return None


# ---------------------------------------------------------------------------------------------
# our arm

def run_ours(args, rank, world, local):
    import numpy as np
    import torch

    from fastwarp_b200 import CudaBackend
    from fastwarp_b200.phantoms import head_pair
    from fastwarp_b200.serve import Server

    shape = tuple(int(x) for x in args.shape.split(",")) if args.shape else SHAPE
    log(f"generating the {shape} phantom pair")
    g, fixed, mg, moving, initial = head_pair(shape, seed=20_260_910 + 2 + rank)
    rec = recipe()
    conc = 1 if args.mode == "sequential" else max(1, args.concurrency)
    b = CudaBackend(local)
    fi, mi = b.upload_image(g, fixed), b.upload_image(mg, moving)

    def batch(server, n, device=True):
        if device:
            ts = [server.submit(rec, g, [fi], mg, [mi], initial, keep_on_device=True)
                  for _ in range(n)]
        else:
            ts = [server.submit(rec, g, [fixed], mg, [moving], initial) for _ in range(n)]
        # a client consumes each result as it arrives: the fields go back to their slot's
        # buffer cache before that slot's next registration needs them (holding every result
        # of the batch instead would grow each slot's memory pool inside the timed region)
        outs = []
        for t in ts:
            o = server.wait(t)
            if o["status"] != 0:
                raise RuntimeError(o["error"])
            Server.free_device_fields(o)
            outs.append(o)
        return outs

    def span_ms(outs):
        return max(o["device_end_ms"] for o in outs) - min(o["device_start_ms"] for o in outs)

    log(f"server with {conc} slots; warm-up")
    srv = Server(local, slots=conc)
    n = args.steps * conc
    # the first warm-up batch has the timed batch's size, so every slot's pool and buffer cache
    # already hold what the timed registrations will use
    for w in range(args.warmup):
        batch(srv, n if w == 0 else conc)
    launches0 = srv.stats()["kernel_launches"]
    graphs0 = srv.stats()["graph_launches"]
    log(f"timed: {n} registrations")
    clocks = Clocks(local)
    torch.cuda.synchronize(local)
    barrier(world)
    clocks.start()
    srv.mark()
    outs = batch(srv, n)
    clk = clocks.stop()
    barrier(world)
    t_dev = span_ms(outs) / 1000.0
    t_max = max_over_ranks(t_dev, world)
    value = sum_over_ranks(n, world) / t_max * 3600.0
    st = srv.stats()
    launches = st["kernel_launches"] - launches0
    graphs = st["graph_launches"] - graphs0
    lat = sorted(o["queued_s"] + o["run_s"] for o in outs)

    def pct(p):
        return lat[min(len(lat) - 1, int(round(p / 100.0 * (len(lat) - 1))))]

    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "registrations/hour",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t_max / args.steps * 1000.0, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded phantom pair, no dataset)",
        "config": {"workload": f"head-1mm SyN stage {shape[0]}x{shape[1]}x{shape[2]} CC r4 "
                               f"shrink 4/2/1 sigma 2/1/0 iters 70/50/20",
                   "mode": args.mode, "slots": conc, "registrations_per_step": conc,
                   "iterations_run": outs[0]["iterations"],
                   "final_cc_energy": outs[0]["final_energy"],
                   "device_bytes_per_registration": outs[0]["device_bytes"],
                   "peak_reserved_bytes": st["peak_reserved_bytes"],
                   "l2_flush": "not needed: working set >> L2",
                   "parallelism": f"replicas x{world}"},
        "latency_s": {"p50": round(pct(50), 4), "p95": round(pct(95), 4),
                      "p99": round(pct(99), 4)},
        "gpu_launches": int(launches), "graph_launches": int(graphs),
    }
    if clk:
        out["clocks"] = clk
    srv.close()
    # the same registrations one at a time on the same kernels (served vs sequential)
    if conc > 1:
        log("sequential comparison")
        seq = Server(local, slots=1)
        batch(seq, 3)
        seq.mark()
        so = batch(seq, max(2, min(n, 2 * conc)))
        t_seq = span_ms(so) / 1000.0
        seq_value = len(so) / t_seq * 3600.0
        seq.close()
        out["config"]["sequential_value"] = round(seq_value, 1)
        out["config"]["served_over_sequential"] = round(value / world / seq_value, 3)
        out["config"]["sequential_latency_s"] = round(statistics.median(
            o["run_s"] for o in so), 4)
        out["config"]["sequential_run_s"] = [round(o["run_s"], 4) for o in so]
        # the reference's execution shape: the loop drives one synchronous Backend op at a time
        from fastwarp_b200.syn import run_syn_ops
        log("op-by-op comparison")
        run_syn_ops(b, rec, g, [fixed], mg, [moving], initial)
        t0 = time.perf_counter()
        run_syn_ops(b, rec, g, [fixed], mg, [moving], initial)
        t_ops = time.perf_counter() - t0
        out["config"]["op_by_op_value"] = round(3600.0 / t_ops, 1)
        out["config"]["served_over_op_by_op"] = round(value / world / (3600.0 / t_ops), 3)
    # per-kernel roofline at the finest level (CUDA events on the engine stream)
    log("kernel timing")
    t = time_kernels(b, fi, b.upload_image(g, fixed), 20)
    # launches per iteration (ncu launch list of a registration: 4 inversions of 1.08 bodies on
    # average, each body its bound, step and fix kernels; the step carries the body's bytes)
    per_iter = {"warp": 2, "cc_pair": 1, "smooth": 2, "compose": 2, "inv_step": 4.3}
    dom = max(per_iter, key=lambda k: t[k][0] * per_iter[k])
    ms, by = t[dom]
    peak, src = peaks()
    achieved = by / (ms / 1000.0) / 1e9
    traffic = None
    kt = kernel_traffic()
    nvox = shape[0] * shape[1] * shape[2]
    if kt and dom in kt.get("dram_bytes_per_voxel", {}):
        traffic = kt["dram_bytes_per_voxel"][dom] * nvox
    out["roofline"] = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1),
                       "peak": peak, "peak_source": f"{src} hbm_gbs (copy, burst)",
                       "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                       "algorithmic_bytes_per_launch": by, "ms_per_launch": round(ms, 4),
                       "kernels_ms": {k: round(v[0], 4) for k, v in t.items()},
                       "kernels_gbs": {k: round(v[1] / (v[0] / 1000.0) / 1e9, 1)
                                       for k, v in t.items()}}
    # end to end through the public host API: host images in (copied at submit), AoS float32
    # fields out; wall clock from the first submit to the last result
    if not args.no_e2e:
        log("end to end")
        e2e = Server(local, slots=conc)
        ne = max(conc, min(n, 2 * conc))
        # warm-up with as many requests in flight as the timed batch: the pinned staging and
        # result buffers (and the slots' device caches) reach their working size before timing
        batch(e2e, ne, device=False)
        t0 = time.perf_counter()
        eo = batch(e2e, ne, device=False)
        te = max_over_ranks(time.perf_counter() - t0, world)
        e2e.close()
        shape3 = int(np.prod([eo[0]["grid"].size[a] for a in range(3)]))
        out["e2e"] = {"value": round(sum_over_ranks(ne, world) / te * 3600.0, 1),
                      "unit": "registrations/hour",
                      "h2d_bytes_per_step": int((fixed.nbytes + moving.nbytes) * conc),
                      "d2h_bytes_per_step": int(2 * 12 * shape3 * conc),
                      "timing": "wall clock, first submit to last result (host copies included)"}
    if not args.no_batch:
        log("batching form (config 4)")
        out["batched"] = batch_leg(b, rank, args.subjects)
    if not args.no_mi:
        log("sampled Mattes MI leg and linear chain")
        out["mattes_mi"] = mi_leg(b, g, fixed, mg, moving, initial, fi, mi, rank, world)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        log("CPU baseline sample")
        out["cpu_baseline"] = cpu_sample(g, fixed, mg, moving, initial, rec, shape)
        if not args.no_mi:
            out["mattes_mi"]["cpu_baseline"] = mi_cpu_baseline(g, fixed, mg, moving, initial)
    b.close()
    return out


# ---------------------------------------------------------------------------------------------
# the CPU engine (oracle restatement of the reference's engine="cpu")

def oracle_inputs(g, fixed, mg, moving, initial, rec):
    import numpy as np

    import oracle as O

    def og(grid):
        return O.make_grid(tuple(grid.size), tuple(grid.spacing), tuple(grid.origin),
                           np.array(grid.direction[:]).reshape(3, 3))

    oaff = O.make_affine(np.array(initial.matrix[:]).reshape(3, 3), tuple(initial.offset))
    r = O.syn_recipe(rec.gradient_step, rec.update_field_variance, rec.total_field_variance,
                     rec.cc_radius, list(rec.iterations), list(rec.shrink_factors),
                     list(rec.smoothing_sigmas), False, rec.convergence_threshold,
                     rec.convergence_window, [1.0])
    return O, r, og(g), og(mg), oaff, fixed.astype(np.float64), moving.astype(np.float64)


# consecutive iterations timed per level (the coarse ones are short and vary more)
SAMPLE_ITERS = [4, 2, 1]


def cpu_sample(g, fixed, mg, moving, initial, rec, shape):
    """A bounded sample of the CPU engine: the level smoothing and a few consecutive SyN
    iterations (state carried from one to the next) per level, timed on the oracle; the
    registration time is each level's smoothing plus its mean iteration time times the recipe's
    iterations, which both engines run in full (threshold -1: 70/50/20)."""
    import numpy as np
    O, r, ofg, omg, oaff, f64, m64 = oracle_inputs(g, fixed, mg, moving, initial, rec)
    iters = list(rec.iterations)
    total = 0.0
    parts = []
    t_all = time.perf_counter()
    for level in range(len(iters)):
        lg = O.syn_level_grid(r, ofg, level)
        t0 = time.perf_counter()
        s = rec.smoothing_sigmas[level]
        fs = O.smooth_recursive(ofg, f64, (s, s, s)) if s > 0 else f64
        ms = O.smooth_recursive(omg, m64, (s, s, s)) if s > 0 else m64
        t_smooth = time.perf_counter() - t0
        shp = O.grid_shape(lg) + (3,)
        state = {k: np.zeros(shp) for k in ("f2m", "f2m_inv", "m2m", "m2m_inv")}
        k = SAMPLE_ITERS[min(level, len(SAMPLE_ITERS) - 1)]
        t0 = time.perf_counter()
        for _ in range(k):
            O.syn_step(r, lg, ofg, [fs], omg, [ms], oaff, state)
        t_it = (time.perf_counter() - t0) / k
        total += t_smooth + iters[level] * t_it
        parts.append(f"L{level} {tuple(lg.size)}: {k} iterations, {t_it:.3f} s/iter")
    sample = time.perf_counter() - t_all
    return {"value": round(3600.0 / total, 3), "unit": "registrations/hour",
            "cores": O.num_threads(), "kind": "port",
            "sample": f"level smoothing + {'/'.join(map(str, SAMPLE_ITERS))} consecutive SyN "
                      f"iterations per level ({sample:.1f} s of CPU work), times the "
                      f"{'/'.join(map(str, iters))} iterations both engines run: " +
                      "; ".join(parts),
            "iterations": iters, "sample_s": round(sample, 2),
            "seconds_per_registration": round(total, 2)}


def cpu_full_registration(g, fixed, mg, moving, initial, rec):
    """One whole registration on the oracle (every iteration), wall clock."""
    O, r, ofg, omg, oaff, f64, m64 = oracle_inputs(g, fixed, mg, moving, initial, rec)
    t0 = time.perf_counter()
    _, _, recs, _ = O.syn_run(r, ofg, [f64], omg, [m64], oaff)
    return time.perf_counter() - t0, len(recs), O.num_threads()


def run_reference(args, rank, world):
    if rank != 0:
        return None
    from fastwarp_b200.phantoms import head_pair
    shape = tuple(int(x) for x in args.shape.split(",")) if args.shape else SHAPE
    g, fixed, mg, moving, initial = head_pair(shape, seed=20_260_910 + 2)
    rec = recipe()
    workload = (f"head-1mm SyN stage {shape[0]}x{shape[1]}x{shape[2]} CC r4 shrink 4/2/1 "
                f"sigma 2/1/0 iters 70/50/20 (all run)")
    engine = ("f64 CPU oracle restating the reference's engine=cpu (the Rust reference cannot "
              "be built here)")
    if args.full_cpu:
        est = cpu_sample(g, fixed, mg, moving, initial, rec, shape)
        secs, n, cores = cpu_full_registration(g, fixed, mg, moving, initial, rec)
        return {"impl": "reference", "mode": "full-cpu", "workload": workload, "engine": engine,
                "seconds_per_registration": round(secs, 2), "iterations": n, "cores": cores,
                "extrapolated_seconds_per_registration": est["seconds_per_registration"],
                "extrapolation_sample": est["sample"]}
    for _ in range(args.warmup if args.warmup < 2 else 1):
        cpu_sample(g, fixed, mg, moving, initial, rec, shape)
    vals, walls = [], []
    last = None
    for _ in range(args.steps):
        t0 = time.perf_counter()
        last = cpu_sample(g, fixed, mg, moving, initial, rec, shape)
        walls.append(time.perf_counter() - t0)
        vals.append(last["value"])
    v = statistics.mean(vals)
    return {
        "impl": "reference", "metric": METRIC, "value": round(v, 3),
        "unit": "registrations/hour", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(statistics.mean(walls) * 1000, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded phantom pair, no dataset)",
        "config": {"workload": workload, "engine": engine,
                   "step": "one bounded sample (level smoothing and a few consecutive SyN "
                           "iterations per level); value = registrations/hour of its measured "
                           "per-iteration times times the 70/50/20 iterations both engines run",
                   "iterations": last["iterations"],
                   "seconds_per_registration": last["seconds_per_registration"]},
        "cpu_baseline": {"value": round(v, 3), "unit": "registrations/hour",
                         "cores": last["cores"], "kind": "port", "sample": last["sample"]},
        "e2e": {"value": round(v, 3), "unit": "registrations/hour", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------------------------
# the affine stage's sampled Mattes MI at the finest level, and the linear chain

def mi_leg(b, g, fixed, mg, moving, initial, fi, mi, rank, world, chain=True):
    """Times the sampled Mattes MI of config 2's finest level (25 % regular sampling, 32 bins)
    and the whole linear chain. Per pass: CUDA events on the engine stream, algorithmic bytes
    16 S + min(4 Nm, 32 S); through the host API: wall clock per evaluation (one read-back)."""
    import numpy as np

    from fastwarp_b200 import CudaLinearEngine, linear_transform
    from fastwarp_b200.backend import linear_recipe, run_linear_chain
    eng = CudaLinearEngine(b)
    level = eng.prepare_level_regular(g, fi, mi, 0.25, 1, 32)
    center = tuple(g.origin[a] + 0.5 * (g.size[a] - 1) * g.spacing[a] for a in range(3))
    # the phantom's own map as the evaluated transform: y = M (x - c) + c + t = M x + offset
    M = np.array(initial.matrix[:]).reshape(3, 3)
    t_vec = np.array(initial.offset[:]) - np.array(center) + M @ np.array(center)
    tr = linear_transform("affine", list(M.ravel()) + list(t_vec), center=center)
    passes = level.time_passes(tr, 50)
    peak, src = peaks()
    v, _ = level.value_and_derivative(tr)
    out = {"samples": level.num_valid(), "value": v}
    for name in ("hist", "deriv"):
        ms, by = passes[name]
        gbs = by / (ms / 1000.0) / 1e9
        out[name] = {"ms": round(ms, 5), "algorithmic_bytes": by, "gbs": round(gbs, 1),
                     "frac": round(gbs / peak, 4)}
    out["finish_ms"] = round(passes["finish"][0], 5)
    out["peak"] = {"gbs": peak, "source": f"{src} hbm_gbs (copy, burst)"}
    # through the host API (one device evaluation and one read-back each)
    for _ in range(3):
        level.value(tr)
        level.value_and_derivative(tr)
    n = 50
    t0 = time.perf_counter()
    for _ in range(n):
        level.value(tr)
    out["value_call_ms"] = round((time.perf_counter() - t0) / n * 1000, 4)
    t0 = time.perf_counter()
    for _ in range(n):
        level.value_and_derivative(tr)
    out["value_and_derivative_call_ms"] = round((time.perf_counter() - t0) / n * 1000, 4)
    level.free()
    if not chain:
        return out
    # the whole linear chain at the config-2 shape
    rigid = linear_recipe(iterations=(500, 250, 100), shrink_factors=(4, 2, 1),
                          smoothing_sigmas=(2.0, 1.0, 0.0))
    affine = linear_recipe(iterations=(500, 250, 100), shrink_factors=(4, 2, 1),
                           smoothing_sigmas=(2.0, 1.0, 0.0))
    run_linear_chain(b, rigid, affine, fi, mi, fi, mi)  # warm-up
    b.synchronize()
    t0 = time.perf_counter()
    chain = run_linear_chain(b, rigid, affine, fi, mi, fi, mi)
    t_chain = time.perf_counter() - t0
    out["linear_chain"] = {"seconds": round(t_chain, 3),
                           "rigid_samples": chain["rigid_samples"],
                           "affine_samples": chain["affine_samples"],
                           "rigid_iterations": chain["rigid_iterations"],
                           "affine_iterations": chain["affine_iterations"],
                           "rigid_best_mi": [round(v, 6) for v in chain["rigid_best"]],
                           "affine_best_mi": [round(v, 6) for v in chain["affine_best"]],
                           "rigid_evaluations": chain["rigid_evaluations"],
                           "affine_evaluations": chain["affine_evaluations"],
                           "initial_ms": round(chain["initial_ms"], 2),
                           "prepare_ms": [round(v, 2) for v in
                                          chain["rigid_prepare_ms"] + chain["affine_prepare_ms"]],
                           "optimize_ms": [round(v, 2) for v in
                                           chain["rigid_optimize_ms"] + chain["affine_optimize_ms"]],
                           "affine_samples_from_rigid": chain["affine_samples_cached"],
                           "recipe": "CoM + rigid + affine, MI 32 bins 25 % regular, shrink "
                                     "4/2/1, sigma 2/1/0 vox, 500/250/100 iterations, 1e-6/10"}
    return out


def batch_leg(b, rank, n_subjects=48):
    """Config 4: `n_subjects` two-channel subjects (T1-like and inverted-contrast T2-like), grid
    dims drawn per axis from 160-240 at 1 mm, each with its own random affine and smooth
    displacement, registered to the 193 x 229 x 193 template: SyN CC r4, shrink 4/2/1, sigma
    2/1/0, 70/50/20 iterations all run, equal channel weights. Batched (fw_batch_syn_run: one
    persistent launch per sub-step over all subjects, each level one graph, autotuned tiles)
    against the same subjects one at a time through the single-registration path and served
    through 4 slots; two subjects' batched fields are compared with their runs alone."""
    import numpy as np

    from fastwarp_b200 import SynRecipe, run_syn_batch, run_syn_device
    from fastwarp_b200.phantoms import BASE_SEED, batch_subjects
    from fastwarp_b200.serve import Server
    g, fixed, subjects = batch_subjects(b, n_subjects, seed=BASE_SEED + 4 + rank)
    r = SynRecipe(gradient_step=0.1, update_field_variance=3.0, total_field_variance=0.0,
                  cc_radius=4, iterations=list(ITERATIONS), shrink_factors=list(SHRINK),
                  smoothing_sigmas=list(SIGMAS), convergence_threshold=-1.0,
                  convergence_window=10, channel_weights=[0.5, 0.5])

    def release(res):
        for x in res.subjects:
            if x is not None:
                x.warp.free()
                x.inverse_warp.free()

    t0 = time.perf_counter()
    first = run_syn_batch(b, r, fixed, subjects, download=False)  # tunes each level's shapes
    t_first = time.perf_counter() - t0
    release(first)
    t0 = time.perf_counter()
    res = run_syn_batch(b, r, fixed, subjects, download=False)
    t_batch = time.perf_counter() - t0
    dev_batch = sum(res.level_ms) / 1000.0
    ok = sum(1 for st in res.statuses if st == 0)
    # two subjects against their runs alone (0.05 mm RMS, 1e-4 final CC is the bar)
    checks = []
    for k in (0, n_subjects - 1):
        moving, initial = subjects[k]
        w, iw, recs = run_syn_device(b, r, fixed, moving, initial)
        got = res.subjects[k]
        a, a0 = b.download_field(got.warp), b.download_field(w)
        ia, ia0 = b.download_field(got.inverse_warp), b.download_field(iw)
        checks.append({"subject": k,
                       "rms_mm": float(np.sqrt(((a - a0) ** 2).sum(-1).mean())),
                       "rms_inverse_mm": float(np.sqrt(((ia - ia0) ** 2).sum(-1).mean())),
                       "max_abs_mm": float(max(np.abs(a - a0).max(), np.abs(ia - ia0).max())),
                       "final_cc": got.iterations[-1]["energy"],
                       "final_cc_alone": recs[-1]["energy"]})
        w.free()
        iw.free()
    release(res)
    # the same subjects one at a time (single-registration graphs), on a sample of 8
    ns = min(8, n_subjects)
    b.synchronize()
    t0 = time.perf_counter()
    for moving, initial in subjects[:ns]:
        w, iw, _ = run_syn_device(b, r, fixed, moving, initial)
        w.free()
        iw.free()
    b.synchronize()
    t_seq = (time.perf_counter() - t0) / ns
    # and served through 4 slots (continuous batching of independent registrations)
    with Server(b.device, slots=4) as srv:
        def served():
            ts = [srv.submit(r, g, fixed, moving[0].grid, moving, initial, keep_on_device=True)
                  for moving, initial in subjects]
            for t in ts:
                o = srv.wait(t)
                Server.free_device_fields(o)
        served()
        t0 = time.perf_counter()
        served()
        t_srv = time.perf_counter() - t0
    sizes = [tuple(m[0].grid.size) for m, _ in subjects]
    return {"workload": f"{n_subjects} two-channel subjects, dims U(160-240) per axis, to the "
                        "193x229x193 template; CC r4 shrink 4/2/1 sigma 2/1/0 70/50/20 (all run)",
            "value": round(n_subjects / t_batch * 3600.0, 1), "unit": "registrations/hour",
            "seconds": round(t_batch, 3), "device_seconds": round(dev_batch, 3),
            "first_run_seconds_with_tuning": round(t_first, 3),
            "subjects_ok": ok,
            "sequential_value": round(3600.0 / t_seq, 1),
            "sequential_seconds_per_subject": round(t_seq, 4),
            "served_4_slots_value": round(n_subjects / t_srv * 3600.0, 1),
            "batched_over_sequential": round(t_seq * n_subjects / t_batch, 3),
            "batched_over_served": round(t_srv / t_batch, 3),
            "level_ms": [round(x, 2) for x in res.level_ms],
            "prepare_ms": [round(x, 2) for x in res.prepare_ms],
            "finish_ms": round(res.finish_ms, 2),
            "tuning": res.tuning, "device_bytes": res.device_bytes,
            "moving_dims_min": [min(x[a] for x in sizes) for a in range(3)],
            "moving_dims_max": [max(x[a] for x in sizes) for a in range(3)],
            "vs_alone": checks}


class MemorySampler:
    """Polls the device's used memory (cudaMemGetInfo through the library) every 50 ms."""

    def __init__(self, device):
        self.device = device
        self.peak = 0
        self.start = self.used()
        self.stop = threading.Event()
        self.thread = threading.Thread(target=self.run, daemon=True)

    def used(self):
        import ctypes as C

        from fastwarp_b200 import _native as N
        free, total = C.c_uint64(), C.c_uint64()
        if N.lib().fw_device_memory(self.device, C.byref(free), C.byref(total)) != 0:
            return 0
        return total.value - free.value

    def run(self):
        while not self.stop.is_set():
            self.peak = max(self.peak, self.used())
            self.stop.wait(0.05)

    def __enter__(self):
        self.thread.start()
        return self

    def __exit__(self, *exc):
        self.stop.set()
        self.thread.join()


def stream_leg(b, rank, rates=(20, 100, 400), n=40, compress=360.0, slots=4, budget=170e9):
    """Config 5: an open-loop request stream, Poisson arrivals at each nominal rate (requests per
    hour), time-compressed by `compress` (one wall second stands for `compress` seconds), 70 %
    single-channel SyN / 20 % affine-only Mattes MI fits / 10 % two-channel SyN, grid dims drawn
    per axis from 160-240 at 1 mm, every request a seeded phantom pair kept on the device.
    Admission by a 170 GB HBM budget. Each stream runs through the server with `slots` slots and
    through one slot (sequential execution of the same stream, the same arrival times);
    reported per rate: throughput, p50/p95/p99 latency (submit to result, wall seconds) and
    peak HBM (admission estimates and measured device use)."""
    import numpy as np

    from fastwarp_b200 import SynRecipe, linear_transform
    from fastwarp_b200.backend import linear_recipe
    from fastwarp_b200.phantoms import BASE_SEED, stream_requests
    from fastwarp_b200.serve import Server
    reqs = stream_requests(b, n, seed=BASE_SEED + 5 + rank)

    def syn_recipe(channels):
        return SynRecipe(gradient_step=0.1, update_field_variance=3.0, total_field_variance=0.0,
                         cc_radius=4, iterations=list(ITERATIONS), shrink_factors=list(SHRINK),
                         smoothing_sigmas=list(SIGMAS), convergence_threshold=-1.0,
                         convergence_window=10, channel_weights=[1.0 / channels] * channels)
    rs = {"syn": syn_recipe(1), "syn2": syn_recipe(2)}
    lr = linear_recipe(iterations=(500, 250, 100), shrink_factors=(4, 2, 1),
                       smoothing_sigmas=(2.0, 1.0, 0.0))

    def submit(srv, q):
        if q["kind"] == "affine":
            g = q["grid"]
            c = tuple(g.origin[a] + 0.5 * (g.size[a] - 1) * g.spacing[a] for a in range(3))
            start = linear_transform("affine", list(np.eye(3).ravel()) + [0.0] * 3, center=c)
            return srv.submit_linear(lr, g, q["fixed"][0], g, q["moving"][0], start)
        return srv.submit(rs[q["kind"]], q["grid"], q["fixed"], q["grid"], q["moving"],
                          q["initial"], keep_on_device=True)

    def wait(srv, q, t):
        if q["kind"] == "affine":
            o = srv.wait_linear(t)
        else:
            o = srv.wait(t)
            Server.free_device_fields(o)
        if o["status"] != 0:
            raise RuntimeError(o["error"])
        return o["queued_s"] + o["run_s"]

    def run(k, arrivals):
        with Server(b.device, budget_bytes=int(budget), slots=k) as srv:
            for q in [next(x for x in reqs if x["kind"] == kd) for kd in ("syn", "affine", "syn2")
                      if any(x["kind"] == kd for x in reqs)]:
                wait(srv, q, submit(srv, q))  # warm-up: each kind once
            sub = [None] * n
            tickets = [None] * n

            def feeder():
                t0 = time.perf_counter()
                for i, q in enumerate(reqs):
                    dt = arrivals[i] - (time.perf_counter() - t0)
                    if dt > 0:
                        time.sleep(dt)
                    sub[i] = time.perf_counter()
                    tickets[i] = submit(srv, q)
            with MemorySampler(b.device) as mem:
                th = threading.Thread(target=feeder)
                th.start()
                lat = []
                for i, q in enumerate(reqs):
                    while tickets[i] is None:
                        time.sleep(0.001)
                    lat.append(wait(srv, q, tickets[i]))
                th.join()
            st = srv.stats()
        span = max(s + l for s, l in zip(sub, lat)) - min(sub)
        lat_sorted = sorted(lat)

        def pct(p):
            return lat_sorted[min(n - 1, int(round(p / 100.0 * (n - 1))))]
        return {"throughput_per_hour_wall": round(n / span * 3600.0, 1),
                "throughput_per_hour_nominal": round(n / span * 3600.0 / compress, 2),
                "p50_s": round(pct(50), 3), "p95_s": round(pct(95), 3), "p99_s": round(pct(99), 3),
                "span_s": round(span, 2), "peak_reserved_bytes": st["peak_reserved_bytes"],
                "peak_device_bytes_above_start": max(0, mem.peak - mem.start)}
    out = {"workload": f"{n} requests per rate, 70/20/10 SyN / affine-only / two-channel SyN, "
                       "dims U(160-240) per axis, SyN CC r4 4/2/1 70/50/20, affine MI 32 bins "
                       "25 % 4/2/1 500/250/100",
           "compress": compress, "budget_bytes": int(budget), "slots": slots,
           "kinds": {kd: sum(1 for q in reqs if q["kind"] == kd) for kd in ("syn", "affine", "syn2")},
           "rates": {}}
    b.release_idle_buffers()  # the generation's temporaries leave the device
    rng = np.random.default_rng(20_260_910 + 55)
    for rate in rates:
        gaps = rng.exponential(3600.0 / (rate * compress), size=n)
        arrivals = np.concatenate([[0.0], np.cumsum(gaps)[:-1]])
        served = run(slots, arrivals)
        seq = run(1, arrivals)
        out["rates"][str(rate)] = {"served": served, "sequential": seq,
                                   "served_over_sequential_throughput": round(
                                       served["throughput_per_hour_wall"] /
                                       seq["throughput_per_hour_wall"], 3)}
    return out


def mi_cpu_baseline(g, fixed, mg, moving, initial):
    """The oracle's sampled Mattes MI value and derivative on the same finest-level samples
    (the reference's MattesMi::evaluate restated, all host cores)."""
    import numpy as np

    import oracle as O
    og = O.make_grid(tuple(g.size), tuple(g.spacing), tuple(g.origin),
                     np.array(g.direction[:]).reshape(3, 3))
    omg = O.make_grid(tuple(mg.size), tuple(mg.spacing), tuple(mg.origin),
                      np.array(mg.direction[:]).reshape(3, 3))
    f64, m64 = fixed.astype(np.float64), moving.astype(np.float64)
    pts = O.sample_points_regular(og, 0.25, 1)
    kept, fbin, binning = O.prepare_samples(og, f64, omg, m64, pts, 32)
    center = tuple(g.origin[a] + 0.5 * (g.size[a] - 1) * g.spacing[a] for a in range(3))
    M = np.array(initial.matrix[:]).reshape(3, 3)
    t_vec = np.array(initial.offset[:]) - np.array(center) + M @ np.array(center)
    t = O.linear_transform("affine", list(M.ravel()) + list(t_vec), center=center)
    O.mi_evaluate(binning, omg, m64, kept, fbin, t)
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        v, _, _, _ = O.mi_evaluate(binning, omg, m64, kept, fbin, t)
    secs = (time.perf_counter() - t0) / reps
    return {"value_and_derivative_ms": round(secs * 1000, 2), "value": v,
            "samples": int(len(fbin)), "cores": O.num_threads(), "kind": "port"}


def main():
    args = parse()
    if args.impl == "reference":
        # one CPU process with no collective: rank 0 runs and prints, the other ranks exit 0 at
        # once (no process group, so no rank waits on rank 0's minutes of CPU work)
        out = run_reference(args, int(os.environ.get("RANK", "0")),
                            int(os.environ.get("WORLD_SIZE", "1")))
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    rank, world, local = dist_init(args)
    if args.only:
        out = run_one_leg(args, rank, world, local)
    elif args.kernels_only:
        out = run_kernels_only(args, local)
    else:
        out = run_ours(args, rank, world, local)
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
