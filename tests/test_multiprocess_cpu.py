"""The N > 1 launch path of bench.py without a GPU: one process per rank over
gloo (torch.distributed), rendezvous on 127.0.0.1. Replicas only — each rank
renders its own sample range and the job's time is the maximum over ranks —
so the host logic under test is the process-group plumbing, the max reduction
and the rank-0-only output of the reference arm."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _allreduce_rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import argparse

    import bench
    ws, r, local, pg = bench.dist_setup(argparse.Namespace())
    assert (ws, r) == (world, rank)
    bench.barrier(pg, local)
    m = bench.allreduce_max(pg, float(10 * rank + 1), local)
    out.put((rank, m))
    dist.destroy_process_group()


def test_allreduce_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    ps = [ctx.Process(target=_allreduce_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 11.0), (1, 11.0)]


def test_reference_arm_under_torchrun_prints_one_line(ref_built):
    port = 30500 + (os.getpid() % 1000)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--width", "64",
           "--height", "32", "--spp", "1", "--n-spheres", "8", "--cpu-seconds", "0.2"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0
