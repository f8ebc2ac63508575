"""Multi-rank host path of bench.py on CPU (gloo, world size 2).

On several GPUs the bench runs one process per GPU, each advancing its own
field (replicas: a domain is never sharded), and reports the whole job's
rate over the slowest rank's time.  These tests run that host logic with
two gloo ranks on 127.0.0.1, and the reference arm under torchrun, where
rank 0 alone prints its line and the other ranks exit without work."""
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


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r took (10 + r) ms for its steps and (50 - r) ms end to end
        got = bench.reduce_max([10.0 + rank, 50.0 - rank], dist, "cpu")
        rate = bench.whole_job_rate(1000, world, 20, got[0])
        q.put((rank, got, rate))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate():
    import torch.multiprocessing as mp
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, rate in res:
        assert got == [11.0, 50.0]  # slowest step time, slowest end-to-end time
        assert rate == pytest.approx(1000 * 2 * 20 / 11e-3)


def test_whole_job_rate_single_rank():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max([3.0, 4.0], None, "cpu") == [3.0, 4.0]
    assert bench.whole_job_rate(100, 1, 10, 2.0) == pytest.approx(100 * 10 / 2e-3)


def test_reference_arm_under_torchrun_prints_once():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--size", "48"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0
