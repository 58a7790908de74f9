"""The continuous-batching job server (dpd_server_* through the C ABI).

Stated tolerances: a job's thermo rows in the mix equal its rows alone within 1e-4
relative over its first 30 steps (the only difference is the FP32 summation order of
forces, which a chaotic trajectory amplifies slowly), and its mean temperature and
pressure agree within 2%; every job finishes; the device memory in use never exceeds
the budget; a job larger than the budget is refused at submission."""
import re

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _jobs():
    from gpumdpd_b200 import inputs
    jobs = inputs.job_stream(n_jobs=6, seed=3, n_min=1000, n_max=12000, steps_min=40, steps_max=120,
                             rate=1.0, thermo=10)
    return [s for _, s, _ in jobs]


def _alone(system):
    from gpumdpd_b200 import Engine
    e = Engine(system.run_in, system=system.c_system())
    steps = int(re.search(r"(?m)^run (\d+)$", system.run_in).group(1))
    e.run(steps)
    th = e.thermo()
    st = e.state()
    e.close()
    return th, st, steps


def test_job_same_alone_and_in_the_mix():
    from gpumdpd_b200.server import Server
    systems = _jobs()
    srv = Server(hbm_budget_bytes=8e9, chunk_steps=16)
    ids = [srv.submit(systems[0]), srv.submit(systems[1])]
    srv.step()  # the first two are on the GPU when the others arrive
    ids += [srv.submit(s) for s in systems[2:]]
    srv.drain()
    for jid, s in zip(ids, systems):
        r = srv.result(jid)
        assert r["status"] == "done", r
        th, st, steps = _alone(s)
        assert r["steps"] == steps
        assert r["last_step"] == th["step"][-1]
        t_mean = th["temp"][1:].mean() if len(th["temp"]) > 1 else th["temp"][0]
        p_mean = th["pressure"][1:].mean() if len(th["pressure"]) > 1 else th["pressure"][0]
        assert r["mean_temp"] == pytest.approx(t_mean, rel=2e-2)
        assert r["mean_pressure"] == pytest.approx(p_mean, rel=2e-2)
        fin = srv.state(jid)
        assert np.isfinite(fin["x"]).all() and np.isfinite(fin["v"]).all()


def test_early_rows_match_alone_run():
    """A short job (30 steps, thermo every step): every row in the mix equals the row alone
    within 1e-4 relative."""
    from gpumdpd_b200 import inputs
    from gpumdpd_b200.server import Server
    probe = inputs.binary_mixture(9.0, 40.0, seed=21, nsteps=30, thermo=1)
    others = _jobs()[:3]
    srv = Server(hbm_budget_bytes=8e9, chunk_steps=7)
    for s in others[:2]:
        srv.submit(s)
    srv.step()
    jid = srv.submit(probe)
    srv.submit(others[2])
    srv.drain()
    th, st, steps = _alone(probe)
    r = srv.result(jid)
    assert r["status"] == "done"
    assert r["last_temp"] == pytest.approx(th["temp"][-1], rel=1e-4)
    assert r["last_pressure"] == pytest.approx(th["pressure"][-1], rel=1e-4)
    assert r["mean_temp"] == pytest.approx(th["temp"][1:].mean(), rel=1e-4)
    assert r["mean_pressure"] == pytest.approx(th["pressure"][1:].mean(), rel=1e-4)
    fin = srv.state(jid)
    L = probe.box
    dx = fin["x"] - st["x"]
    dx -= L * np.round(dx / L)
    assert np.abs(dx).max() < 1e-3


def test_budget_admission_and_release():
    """A budget that holds about two of the jobs: the rest wait in the queue, memory in use
    stays within the budget, and every job finishes."""
    from gpumdpd_b200.server import Server
    from gpumdpd_b200 import capi
    systems = _jobs()
    # size the budget from the device memory of the two largest jobs running together
    big = sorted(systems, key=lambda s: -s.n)[:2]
    probe = Server(hbm_budget_bytes=64e9, chunk_steps=1)
    for s in big:
        probe.submit(s)
    probe.step()
    two = probe.stats()["device_bytes"]
    probe.drain()
    probe.close()
    budget = 1.05 * two
    srv = Server(hbm_budget_bytes=budget, chunk_steps=32)
    ids = [srv.submit(s) for s in systems]
    saw_queue = False
    for _ in range(10 ** 6):
        a, q = srv.step()
        assert srv.stats()["device_bytes"] <= budget
        saw_queue |= q > 0
        if a == 0 and q == 0:
            break
    assert saw_queue
    res = [srv.result(j) for j in ids]
    assert all(r["status"] == "done" for r in res)
    assert srv.stats()["device_bytes"] == 0
    assert srv.stats()["particle_steps"] == sum(s.n * r["steps"] for s, r in zip(systems, res))
    with pytest.raises(capi.DpdError) as ex:
        tiny = Server(hbm_budget_bytes=1e5, chunk_steps=8)
        tiny.submit(systems[0])
    assert ex.value.code == -4


def test_rdf_of_a_served_job():
    from gpumdpd_b200 import inputs
    from gpumdpd_b200.server import Server
    s = inputs.binary_mixture(10.0, 35.0, seed=4, nsteps=60, thermo=20, rdf=(3.0, 60, 10))
    srv = Server(hbm_budget_bytes=4e9, chunk_steps=25)
    jid = srv.submit(s)
    srv.drain()
    g, ns = srv.rdf(jid, 60)
    assert ns >= 6
    assert np.isfinite(g).all()
    assert g[-10:].mean() == pytest.approx(1.0, abs=0.15)


def test_jobs_with_fixes_and_walls_in_the_mix():
    """Jobs with group fixes (spring, rvcm, recenter) and particle walls (move, two_wall)
    share a cohort with a plain job: each finishes with the state of its run alone, to
    FP32 summation order after 20 steps."""
    from gpumdpd_b200 import inputs
    from gpumdpd_b200.server import Server
    systems = [inputs.probe_fixes(L=9.0, seed=5, nsteps=20, thermo=5, spring_file=None),
               inputs.wall_channel(L=8.0, Lz=12.0, seed=6, nsteps=20, thermo=5),
               inputs.plain_dpd(L=7.0, seed=7, nsteps=20, thermo=5)]
    srv = Server(hbm_budget_bytes=8e9, chunk_steps=8)
    ids = [srv.submit(s) for s in systems]
    srv.drain()
    for jid, s in zip(ids, systems):
        r = srv.result(jid)
        assert r["status"] == "done", r
        _, st, steps = _alone(s)
        assert r["steps"] == steps
        fin = srv.state(jid)
        L = s.hi - s.lo
        dx = fin["x"] - st["x"]
        dx -= L * np.round(dx / L)
        assert np.abs(dx).max() < 1e-3
        assert np.abs(fin["v"] - st["v"]).max() < 1e-2
