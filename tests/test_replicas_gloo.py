"""bench.py's multi-GPU path is replicas only: every rank advances its own
model and the job's throughput is all ranks' work over the slowest rank's
time.  The rank logic (process group, barrier, max over ranks) runs here as
two gloo processes on the CPU."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, ws, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(ws),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup("gloo")
    try:
        bench.barrier(w)
        t = [0.5, 2.0][r]                      # rank 1 is the slow one
        v = bench.replica_throughput(w, 1000.0, t)
        out.put((r, bench.allmax(w, float(r + 1)), v))
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    for r, mx, v in got:
        assert mx == 2.0
        assert v == pytest.approx(2 * 1000.0 / 2.0)
