"""The multi-rank (torchrun) paths of bench.py, on CPU with gloo at world size 2.

The ISPH-DEM step has no cross-GPU exchange, so ranks are independent
replicas.  What has to hold across ranks: every rank reaches the same
collectives (barriers, the max-over-ranks time, the sum of particles), only
rank 0 prints, and the reference arm runs on rank 0 alone while the other
ranks exit 0 without work.
"""
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


def _reduce_worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.reduce_over_ranks(dist, 10.0 + 5.0 * rank, "max")
        n = bench.reduce_over_ranks(dist, 100 + rank, "sum")
        q.put((rank, t, n))
    finally:
        dist.destroy_process_group()


def test_reduce_over_ranks_gloo_world2():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_reduce_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 15.0, 201.0), (1, 15.0, 201.0)]


def test_reduce_without_process_group_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.reduce_over_ranks(None, 3.5, "max") == 3.5


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_world2():
    """torchrun --nproc-per-node 2 bench.py --impl reference: rank 0 alone
    times the CPU baseline (the host build of the reference's kernels when it
    was built, else the oracle port) and prints one JSON line; rank 1 exits 0."""
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = "2"
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--no-ref-cuda"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    host_ref = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libsophia_ref_host.so"))
    assert d["cpu_baseline"]["kind"] == ("reference" if host_ref else "port")
    assert d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["config"]["n_sph"] == 301760 and d["config"]["n_dem"] == 20000
    assert str(d["config"]["n_sph"]) in d["cpu_baseline"]["sample"], "the sample must be the whole bed"
    assert d["config"]["parallelism"] == "replicas x2"


@pytest.mark.timeout(600)
def test_column_reference_arm():
    """bench.py --workload column --impl reference: the CPU port on the 3-D
    ISPH column (PCG to 1e-6) prints one JSON line of the same metric."""
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = "2"
    cmd = [sys.executable, "bench.py", "--workload", "column", "--impl", "reference", "--steps", "1",
           "--warmup", "0", "--cpu-seconds", "1"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and "column" in d["metric"]
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
