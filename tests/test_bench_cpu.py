"""CPU tests of bench.py's multi-rank scaffolding: max-over-ranks timing with
world_size 2 on gloo, the weak-scaling aggregate, and the reference arm under
torchrun (rank 0 prints one line, the other rank exits quietly)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    got = bench.max_over_ranks(10.0 + 5.0 * rank, world, device="cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got))


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=5) for _ in range(2))
    assert res == {0: 15.0, 1: 15.0}


def test_weak_throughput():
    import bench
    # 2 ranks, 3 steps of 1 GB each in the slowest rank's 1.5 s -> 4 GB/s
    assert bench.weak_throughput(1e9, 3, 2, 1500.0) == pytest.approx(4.0)
    assert bench.max_over_ranks(7.0, 1) == 7.0


@pytest.mark.slow
def test_reference_arm_under_torchrun_two_ranks():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
