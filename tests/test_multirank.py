"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2): the path runs as
independent replicas (no data-path collective); the job's step time is the max over
ranks and the throughput counts every rank's work."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    local = 0.010 * (rank + 1)          # rank 1 is the slow one
    value, step = bench.replica_throughput(local, 1_000_000, world, torch.device("cpu"))
    q.put((rank, value, step))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_throughput_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, step in res:
        assert step == pytest.approx(0.020)
        assert value == pytest.approx(2 * 1_000_000 / 0.020)


def test_single_rank_is_local_time():
    import bench
    v, s = bench.replica_throughput(0.5, 100, 1, torch.device("cpu"))
    assert s == 0.5 and v == 200


def test_reference_arm_under_torchrun_two_ranks():
    """bench.py --impl reference launched as the multi-GPU runs launch it (torchrun,
    world size 2, here over gloo): rank 0 alone times the reference's CPU path and
    prints one JSON line; rank 1 exits 0 without work."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                          "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py",
                          "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--config", "0"],
                         cwd=root, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["value"] > 0 and line["n_gpus"] == 2
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
