"""Failure paths made on the host, none of which faults or hangs the GPU.

The reference ends the process on any error (CUDA_CHECK -> exit(1),
src/main/common.cuh:46-60).  Here:
- a non-finite state handed in through dpd_set_state (a NaN velocity, a NaN position, a
  velocity of 1e30 that overflows within a few steps) makes dpd_run return
  DPD_E_NUMERIC, and the engine keeps answering;
- inside a server batch the same error fails that job alone: its cohort mates finish
  with their alone-run results (thermo rows within 1e-4 relative over 30 steps, the
  tolerance of the server's alone-vs-mix test);
- a job cancelled while running is frozen, its cohort mates run on unchanged, and its
  batch's device memory returns to the budget once nothing else runs in it; a queued job
  cancelled never starts.
"""
import re

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DPD_E_NUMERIC = -7
DPD_E_CANCELLED = -9


def _alone(system):
    from gpumdpd_b200 import Engine
    e = Engine(system.run_in, system=system.c_system())
    steps = int(re.search(r"(?m)^run (\d+)$", system.run_in).group(1))
    e.run(steps)
    th = e.thermo()
    e.close()
    return th


def _with_v(system, v):
    from gpumdpd_b200 import inputs
    return inputs.System(system.lo, system.hi, system.masses, system.types, system.x, v,
                         bonds=system.bonds, n_bondtypes=system.n_bondtypes, mol=system.mol,
                         run_in=system.run_in, atom_style=system.atom_style)


@pytest.mark.parametrize("what", ["nan_velocity", "nan_position", "huge_velocity"])
def test_nonfinite_state_reports_numeric(what):
    from gpumdpd_b200 import Engine, capi, inputs
    s = inputs.plain_dpd(L=8.0, seed=31, nsteps=50, thermo=5)
    e = Engine(s.run_in, system=s.c_system())
    e.run(3)
    st = e.state()
    x, v = st["x"].copy(), st["v"].copy()
    if what == "nan_velocity":
        v[17, 1] = np.nan
    elif what == "nan_position":
        x[5, 2] = np.nan
    else:
        v[17] = 1.0e30
    e.set_state(x, v)
    with pytest.raises(capi.DpdError) as ex:
        e.run(20)
    assert ex.value.code == DPD_E_NUMERIC, str(ex.value)
    # the engine still answers: its state can be read back
    st2 = e.state()
    assert st2["x"].shape == x.shape
    e.close()
    # and the GPU context is intact: a fresh engine runs a clean system
    e2 = Engine(s.run_in, system=s.c_system())
    e2.run(5)
    assert np.isfinite(e2.thermo()["temp"]).all()
    e2.close()


def test_nonfinite_job_fails_alone_in_its_batch():
    from gpumdpd_b200 import inputs
    from gpumdpd_b200.server import Server
    mates = [inputs.binary_mixture(9.0, 40.0, seed=21, nsteps=30, thermo=1),
             inputs.binary_mixture(8.0, 30.0, seed=22, nsteps=30, thermo=1)]
    bad = inputs.binary_mixture(8.5, 35.0, seed=23, nsteps=30, thermo=1)
    v = bad.v.copy()
    v[3, 0] = np.nan
    bad = _with_v(bad, v)
    srv = Server(hbm_budget_bytes=8e9, chunk_steps=7)
    ids = [srv.submit(mates[0]), srv.submit(bad), srv.submit(mates[1])]
    # all three are queued before the first scheduling point: one cohort (same length)
    for _ in range(10 ** 6):
        try:
            a, q = srv.step()
        except Exception as e:  # the failing job's error is reported by the step
            assert "non-finite" in str(e), str(e)
            continue
        if a == 0 and q == 0:
            break
    rb = srv.result(ids[1])
    assert rb["code"] == DPD_E_NUMERIC, rb
    for jid, s in ((ids[0], mates[0]), (ids[2], mates[1])):
        r = srv.result(jid)
        assert r["status"] == "done", r
        th = _alone(s)
        assert r["last_temp"] == pytest.approx(th["temp"][-1], rel=1e-4)
        assert r["last_pressure"] == pytest.approx(th["pressure"][-1], rel=1e-4)
        assert r["mean_temp"] == pytest.approx(th["temp"][1:].mean(), rel=1e-4)
        assert r["mean_pressure"] == pytest.approx(th["pressure"][1:].mean(), rel=1e-4)
    assert srv.stats()["device_bytes"] == 0


def test_cancel_running_and_queued_jobs():
    from gpumdpd_b200 import inputs
    from gpumdpd_b200.server import Server
    probe = inputs.binary_mixture(9.0, 40.0, seed=21, nsteps=30, thermo=1)
    mate = inputs.binary_mixture(8.0, 30.0, seed=24, nsteps=31, thermo=1)   # same cohort as probe
    long_job = inputs.binary_mixture(10.0, 35.0, seed=25, nsteps=300, thermo=10)  # a cohort alone
    srv = Server(hbm_budget_bytes=8e9, chunk_steps=4)
    ids = [srv.submit(probe), srv.submit(mate), srv.submit(long_job)]
    srv.step()
    b_all = srv.stats()["device_bytes"]
    assert b_all > 0
    srv.cancel(ids[1])
    srv.cancel(ids[2])
    assert srv.result(ids[1])["code"] == DPD_E_CANCELLED
    with pytest.raises(Exception):
        srv.cancel(ids[2])  # already ended
    # the long job's batch holds nothing else: its memory returns to the budget while the
    # probe's batch is still running
    released = False
    for _ in range(10 ** 6):
        a, q = srv.step()
        if a > 0 and srv.stats()["device_bytes"] < b_all:
            released = True
        if a == 0 and q == 0:
            break
    assert released
    assert srv.stats()["device_bytes"] == 0
    assert srv.result(ids[2])["code"] == DPD_E_CANCELLED
    r = srv.result(ids[0])
    assert r["status"] == "done", r
    th = _alone(probe)
    assert r["last_temp"] == pytest.approx(th["temp"][-1], rel=1e-4)
    assert r["mean_pressure"] == pytest.approx(th["pressure"][1:].mean(), rel=1e-4)
    srv.close()

    # a queued job: a budget that holds one job at a time
    one = Server(hbm_budget_bytes=64e9, chunk_steps=8)
    one.submit(probe)
    one.step()
    b1 = one.stats()["device_bytes"]
    one.drain()
    one.close()
    srv = Server(hbm_budget_bytes=1.2 * b1, chunk_steps=8)
    j1 = srv.submit(probe)
    j2 = srv.submit(probe)
    a, q = srv.step()
    assert (a, q) == (1, 1)
    srv.cancel(j2)
    assert srv.result(j2)["status"] == "cancelled"
    srv.drain()
    assert srv.result(j1)["status"] == "done"
    assert srv.result(j2)["status"] == "cancelled"
