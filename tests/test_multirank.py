"""The bench's multi-rank host logic on CPU ranks (gloo, world size 2): the
rank rendezvous, the max-over-ranks timing and the barrier, and the
reference arm's rule that only rank 0 works and prints. With one process per
GPU, N GPUs run N independent replicas of the step (no data-path
collective); these are the only cross-rank operations."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist

    w, r, _ = bench.dist_setup(None)
    assert (w, r) == (world, rank) and dist.get_backend() == "gloo"
    m = bench.max_over_ranks(w, 1.5 + r)
    bench.barrier(w)
    out.put((r, m))
    dist.destroy_process_group()


def test_max_over_ranks_and_barrier_on_gloo():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = dict(q.get(timeout=5) for _ in range(2))
    assert got == {0: 2.5, 1: 2.5}


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "2000", "--views", "1",
           "--steps", "1", "--warmup", "0"]
    outs = []
    for rank in (1, 0):
        e = dict(env, RANK=str(rank), LOCAL_RANK=str(rank))
        r = subprocess.run(cmd, env=e, capture_output=True, text=True, timeout=600, cwd=ROOT)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(r.stdout.strip())
    assert outs[0] == ""  # rank 1: no work, no line
    line = json.loads(outs[1].splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("port", "reference")
    assert line["e2e"]["h2d_bytes_per_step"] == 0
