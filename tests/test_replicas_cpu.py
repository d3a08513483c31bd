"""CPU tests of bench.py's multi-process (replicas) path over gloo, world size 2.

The hot path has no cross-GPU exchange, so N GPUs run N independent replicas:
the only collectives are the barrier and the max-over-ranks of the timings,
and the reference arm runs on rank 0 alone.
"""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import argparse

    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup(argparse.Namespace(impl="reference"))
    assert (w, r) == (world, rank)
    bench.barrier(w)
    got = bench.max_over_ranks(10.0 + rank, w)
    q.put((rank, got))
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    res = dict(q.get(timeout=5) for _ in range(2))
    assert res == {0: 11.0, 1: 11.0}


def test_reference_arm_prints_once_under_torchrun():
    from oracle.cpu import Reference
    if not Reference.available():
        pytest.skip("reference CPU library not built")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={_free_port()}", str(ROOT / "bench.py"), "--impl",
           "reference", "--gpus", "2", "--scale", "10", "--steps", "2", "--warmup", "1"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
