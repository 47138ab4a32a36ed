"""Host logic of the multi-rank benchmark on CPU: two gloo ranks (world_size 2), each with its own
replica domain, agree on the job time (the maximum over ranks) and on the whole-job value; the
reference arm runs on rank 0 only and the other rank exits cleanly."""
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [12.5, 17.0][rank]  # rank 1 is the slow one
        m = bench.reduce_max(ms, world, "cpu")
        out[rank] = (m, bench.whole_job_value(1000, 10, world, m))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_value():
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1]
    m, v = res[0]
    assert m == 17.0
    assert abs(v - 2 * 1000 * 10 / 0.017) < 1e-6 * v


def test_reference_arm_under_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus",
           "2", "--steps", "1", "--warmup", "0", "--nx", "24", "--ny", "20", "--kmax", "4", "--M", "2"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout  # rank 0 alone prints
    assert '"impl": "reference"' in lines[0]
