"""The N>1 plumbing of bench.py on CPU: two gloo ranks on 127.0.0.1.

The path does not shard: N GPUs run N independent replicas and only the timing crosses ranks
(the max of the per-rank device spans, the sum of the registrations). These tests run those
helpers on two gloo processes, and run the reference arm under torchrun with two ranks, where
rank 0 alone does the CPU work and prints one JSON line and rank 1 exits 0 without work.
"""
import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        span = 1.0 + rank            # per-rank device span in seconds
        regs = 4                     # registrations each replica ran
        t = bench.max_over_ranks(span, world)
        n = bench.sum_over_ranks(regs, world)
        q.put((rank, t, n, n / t * 3600.0))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_time_and_the_summed_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t, n, v in got:
        assert t == 2.0 and n == 8.0           # slowest rank's span, all ranks' registrations
        assert abs(v - 8 / 2.0 * 3600.0) < 1e-9  # whole-job registrations/hour


def test_reference_arm_under_torchrun_prints_one_line_from_rank_0():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py",
           "--impl", "reference", "--gpus", "2", "--shape", "20,24,20", "--steps", "1",
           "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["n_gpus"] == 2 and out["value"] > 0
    assert out["e2e"]["h2d_bytes_per_step"] == 0 and out["cpu_baseline"]["kind"] == "port"
