"""Multi-process paths on CPU (gloo, world size 2): bench.py runs one
independent replica per GPU, reduces the timed region to the slowest rank
and reports the whole-job throughput; its reference arm runs on rank 0 only.
"""
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    my_ms = [1000.0, 1500.0][rank]                 # rank 1 is the slow replica
    mx = bench.reduce_max(my_ms, dist, "cpu")
    thr = bench.job_throughput(5, world, mx)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, mx, thr))


def test_replicas_reduce_to_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, thr in res:
        assert mx == 1500.0                        # both ranks agree on the max
        assert abs(thr - 5 * 2 / 1.5) < 1e-12      # 10 solves in 1.5 s


def test_reference_arm_only_rank0_prints():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--lattice", "4,4,4,4",
                        "--steps", "1", "--warmup", "0", "--cpu-iters", "2"], env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_rank0_line():
    import json
    env = dict(os.environ, RANK="0", LOCAL_RANK="0", WORLD_SIZE="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--lattice", "4,4,4,4",
                        "--steps", "1", "--warmup", "0", "--cpu-iters", "2"], env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["e2e"]["h2d_bytes_per_step"] == 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refqop
    # the reference's own compiled path where oracle/_ref was built, else the port
    assert line["cpu_baseline"]["kind"] == ("reference" if refqop.available() else "port")
    assert line["cpu_baseline"]["cores"] >= 1 and line["value"] is None
