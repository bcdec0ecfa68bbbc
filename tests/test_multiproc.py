"""The N>1 path of bench.py on CPU: replicas joined by torch.distributed (gloo, world_size 2).

bench.py runs one independent sweep per rank (the path does not shard, so no collective
touches the data); ranks only meet to start and stop the timed region together and to take
the max of their times.  These tests run those helpers in two gloo processes, and the
reference arm under torchrun with two ranks (rank 0 measures, rank 1 exits cleanly)."""

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


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench

    w, r, _ = bench.dist_setup()
    try:
        bench.dist_barrier(w)
        q.put((r, bench.dist_max(float(10 * (r + 1)), w)))
    finally:
        import torch.distributed as dist

        dist.destroy_process_group()


def test_gloo_max_and_barrier_two_ranks():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(2))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == {0: 20.0, 1: 20.0}


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={port}", str(ROOT / "bench.py"), "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--workload", "single"]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=580, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
