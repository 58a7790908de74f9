"""Multi-rank host logic on CPU (gloo, two ranks; unmeasured on GPU hardware, since every
run of this build has one GPU):
- bench.py: each rank times its own replica (replicas only; no data-path collective); the
  whole-job value is the sum of the ranks' particles times the steps over the slowest
  rank's time, and both ranks agree on it;
- gpumdpd_b200.shard: a replica sweep spread over the ranks by cost, each rank running its
  own share (here with the FP64 oracle standing in for a rank's GPU), gathers on every rank
  into exactly the single-rank results."""
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


def _sweep():
    from gpumdpd_b200 import inputs
    return inputs.replica_sweep(n_rep=7, L_min=3.2, L_max=5.0, seed=5, nsteps=4, rdf=None, skin=0.0, thermo=1)


def _run_share(systems, share):
    """Each replica of the share: 4 velocity-Verlet steps in the FP64 oracle (a stand-in
    for the rank's packed GPU batch); result = last thermo row (T, P)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle
    out = {}
    for k in share:
        s = systems[k]
        ff = oracle.ff_from_run_in(s.run_in, s.masses)
        o = oracle.run(ff, np.arange(1, s.n + 1), s.types, s.x, s.v, s.lo, s.box, 1, 4, 1)
        out[k] = (float(o["thermo"]["temp"][-1]), float(o["thermo"]["pressure"][-1]))
    return out


def _shard_rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    from gpumdpd_b200 import shard
    w, r, _ = bench.dist_setup(None, backend="gloo")
    systems = _sweep()
    costs = [s.n * 4 for s in systems]
    mine = shard.assign(costs, w)[r]
    res = shard.run_sharded(systems, costs, lambda share: _run_share(systems, share), w, r)
    out.put((r, mine, res))
    bench.barrier(w)
    dist.destroy_process_group()


def test_sweep_sharded_over_two_gloo_ranks_equals_one_rank():
    from gpumdpd_b200 import shard
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    systems = _sweep()
    costs = [s.n * 4 for s in systems]
    # the split: every replica once, on the rank `assign` names, loads within one replica
    shares = [g[1] for g in got]
    assert sorted(shares[0] + shares[1]) == list(range(len(systems)))
    assert shares == shard.assign(costs, 2)
    loads = [sum(costs[k] for k in sh) for sh in shares]
    assert abs(loads[0] - loads[1]) <= max(costs)
    # both ranks gathered the single-rank results exactly
    single = shard.run_sharded(systems, costs, lambda share: _run_share(systems, share), 1, 0)
    for _, _, res in got:
        assert res == single
