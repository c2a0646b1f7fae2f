"""The bench's multi-rank path on the CPU: world size 2 over gloo.

bench.py runs N independent replicas (one per GPU); the only cross-rank steps
are barriers and the max-over-ranks reduction of the timed intervals.  These
tests run that reduction on two gloo ranks, and the reference arm launched as
torchrun would launch it for N = 2 (rank 0 measures and prints, rank 1 exits
cleanly)."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, values, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    assert bench.env_rank() == (rank, rank, world)
    got = bench.max_over_ranks(values[rank], dist, device="cpu")
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, got))


def test_max_over_ranks_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    values = [3.25, 7.5]
    ps = [ctx.Process(target=_rank, args=(r, 2, port, values, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: 7.5, 1: 7.5}
    assert __import__("bench").max_over_ranks(4.0) == 4.0


def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference", "--gpus",
           "2", "--steps", "1", "--warmup", "1", "--lattice-steps", "2"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
