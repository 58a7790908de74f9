"""Multi-rank host logic of bench.py on CPU: two gloo ranks, each timing its own replica
(replicas only; no data-path collective).  The whole-job value is the sum of the ranks'
particles times the steps over the slowest rank's time, and both ranks agree on it."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup(None, backend="gloo")
    assert (w, r) == (world, rank)
    bench.barrier(w)
    local_ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
    value, total = bench.job_value(1000, 20, local_ms, w)
    out.put((rank, value, total))
    bench.barrier(w)
    dist.destroy_process_group()


def test_two_gloo_ranks_report_the_whole_job():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for _, value, total in res:
        assert total == pytest.approx(150.0)
        assert value == pytest.approx(2 * 1000 * 20 / 0.150)
