"""Multi-process plumbing of bench.py on CPU (gloo, world size 2).

The single-case time step does not shard: N GPUs run N independent replicas
and only the timing crosses ranks (max over ranks).  These tests run that
reduction with two gloo ranks, and the reference arm under torchrun, where
rank 0 alone prints the JSON line and the other rank exits 0 without work.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, times, out):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    m = bench.max_over_ranks(dist, times[rank], torch.device("cpu"))
    v = bench.replica_throughput(world, 1000, 10, m)
    out.put((rank, m, v))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    times = [3.5, 7.25]
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, v in res:
        assert m == 7.25                                   # the slowest rank sets the time
        assert v == pytest.approx(2 * 1000 * 10 / 7.25e-3)  # both replicas' cells count


def test_reference_arm_torchrun_world2(tmp_path):
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
           "--config", "viv_cylinder_384x256", "--cpu-seconds", "0.1"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(tmp_path), env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
