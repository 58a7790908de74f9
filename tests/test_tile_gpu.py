"""Pair schedule 11, the cell-tile kernel (no neighbour list), against the FP64 oracle.

Tolerances as for every force test: largest per-particle error within 1e-5 of the RMS
force, at step 0 and at every one of 10 later steps on the engine's own state; thermo
PE and pressure of the log step as the oracle's (1e-6 and 2e-5 relative).  Covered:
tile edges 1-6 and the engine's choice; boxes of 3 and 4 cells per dimension, where a
tile's neighbourhood wraps onto itself; per-type cutoffs; bonds; skins above 0, where
the cells of the last build serve several steps; a staging capacity so small that
every tile falls back to one home cell at a time; several replicas in one batch; the
neighbour set of the current state, built on demand.
"""
import re

import numpy as np
import pytest

from conftest import force_err, load_golden

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _systems():
    from gpumdpd_b200 import inputs, tune
    dpd = inputs.plain_dpd(L=10.0, seed=2024)
    dpd.run_in = tune.with_skin(dpd.run_in, 0.0)
    melt = inputs.diblock_melt(L=12.0, seed=5, nsteps=10, skin=0.0)
    return {
        "dpd_skin0": dpd,
        "dpd_skin03": inputs.plain_dpd(L=10.0, seed=2025),
        "melt_skin0": melt,
        "box4": inputs.binary_mixture(4.5, 35.0, seed=3, skin=0.0),  # 4 cells per dimension
        "box3": inputs.binary_mixture(3.6, 35.0, seed=4, skin=0.0),  # 3 cells per dimension
    }


def _golden(name):
    from gpumdpd_b200.inputs import System
    g = load_golden(name)
    x = np.column_stack([g[f"s0_{c}"] for c in "xyz"])
    v = np.column_stack([g[f"s0_v{c}"] for c in "xyz"])
    lines = [ln for ln in str(g["run_in"]).splitlines() if not ln.startswith("dump")]
    style = "bond" if "bonds" in g else "atomic"
    return System(g["lo"], g["hi"], g["masses"], g["s0_type"], x, v, bonds=g.get("bonds"),
                  n_bondtypes=1 if "bonds" in g else 0, run_in="\n".join(lines) + "\n", atom_style=style)


def _engine(s, **tuning):
    from gpumdpd_b200 import Engine
    e = Engine(s.run_in, system=s.c_system())
    e.set_tuning(pair_variant=11, **tuning)
    return e


def _box(e):
    c = e.cells()
    return c["nc"].astype(np.float64) * c["w"].astype(np.float64)


def _step0(oracle_mod, s, **tuning):
    e = _engine(s, **tuning)
    e.run(0)
    st = e.state()
    ff = oracle_mod.ff_from_run_in(s.run_in, s.masses)
    o = oracle_mod.forces(ff, np.arange(1, s.n + 1), s.types, st["x"], st["v"], s.lo, _box(e), 0, bonds=s.bonds)
    th = e.thermo()
    e.close()
    return st, o, th


@pytest.mark.parametrize("tile", [0, 1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("name", ["dpd_skin0", "melt_skin0", "box3", "box4", "dpd_skin03"])
def test_tile_step0_forces(oracle_mod, name, tile):
    s = _systems()[name]
    st, o, th = _step0(oracle_mod, s, tile=tile)
    assert force_err(st["f"], o["f"]) < TOL
    assert th["pair_pe"][0] == pytest.approx(o["pair_pe"], rel=1e-6)
    assert th["bond_pe"][0] == pytest.approx(o["bond_pe"], rel=1e-6, abs=1e-9)


@pytest.mark.parametrize("name", ["diblock", "mix_rc", "dpd_c1", "dpd_random_only"])
def test_tile_golden_systems(oracle_mod, name):
    s = _golden(name)
    st, o, th = _step0(oracle_mod, s)
    assert force_err(st["f"], o["f"]) < TOL
    g = load_golden(name)
    f_ref = np.column_stack([g[f"s0_f{c}"] for c in "xyz"])
    assert force_err(st["f"], f_ref) < TOL
    assert th["pressure"][0] == pytest.approx(g["thermo_pressure"][0], rel=2e-5)


def test_tile_capacity_fallback(oracle_mod):
    """A staging capacity below a 4^3 tile's neighbourhood (about 540 particles here) but
    above a single cell's (about 54): every tile takes its home cells one at a time."""
    s = _systems()["melt_skin0"]
    st, o, th = _step0(oracle_mod, s, tile=4, tile_capacity=128)
    assert force_err(st["f"], o["f"]) < TOL
    assert th["bond_pe"][0] == pytest.approx(o["bond_pe"], rel=1e-6)


@pytest.mark.parametrize("log", [False, True])
@pytest.mark.parametrize("name", ["dpd_skin0", "melt_skin0", "dpd_skin03"])
def test_tile_forces_every_step(oracle_mod, name, log):
    """Steps 51-60 on the engine's own state; log=False runs the non-log kernel (thermo
    every 1000 steps), log=True the log-step kernel at every step (thermo every step)."""
    s = _systems()[name]
    s.run_in = re.sub(r"(?m)^thermo \d+$", "thermo 1" if log else "thermo 1000", s.run_in)
    e = _engine(s)
    e.run(50)
    ff = oracle_mod.ff_from_run_in(s.run_in, s.masses)
    tags = np.arange(1, s.n + 1)
    dt = float(re.search(r"(?m)^timestep (\S+)$", s.run_in).group(1))
    m = np.asarray(s.masses)[np.asarray(s.types) - 1][:, None]
    for k in range(1, 11):
        e.run(1)
        got = e.state()
        vh = got["v"] - 0.5 * dt * got["f"] / m
        o = oracle_mod.forces(ff, tags, s.types, got["x"], vh, s.lo, _box(e), 50 + k, bonds=s.bonds)
        assert force_err(got["f"], o["f"]) < TOL, k
        if log:
            th = e.thermo()
            assert th["step"][-1] == 50 + k
            assert th["pair_pe"][-1] == pytest.approx(o["pair_pe"], rel=1e-5)
    e.close()


@pytest.mark.parametrize("name", ["dpd_skin0", "box3", "dpd_skin03"])
def test_tile_neighbor_set_on_demand(oracle_mod, name):
    s = _systems()[name]
    e = _engine(s)
    e.run(3)
    c = e.cells()
    got = e.neighbors()
    ref = oracle_mod.pairs_f32(np.arange(1, s.n + 1), c["cell"], c["offset"], c["nc"], c["w"], c["cut2"])
    assert len(got) == len(set(map(tuple, got.tolist())))
    assert set(map(tuple, got.tolist())) == set(map(tuple, ref.tolist()))
    e.close()


def test_tile_batch_of_uneven_replicas(oracle_mod):
    from gpumdpd_b200 import Batch, inputs, tune
    systems = [inputs.binary_mixture(L, a, seed=40 + k, nsteps=10, thermo=1)
               for k, (L, a) in enumerate([(5.0, 25.0), (9.3, 32.0), (13.7, 45.0), (3.5, 40.0)])]
    for s in systems:
        s.run_in = tune.with_skin(s.run_in, 0.0)
    b = Batch([s.run_in for s in systems], [s.c_system() for s in systems],
              tuning={"pair_variant": 11})
    b.run(0)
    for k, s in enumerate(systems):
        st = b.state(k)
        L = np.asarray(s.box)
        nc = np.floor(L)
        Lb = nc * (L / nc).astype(np.float32).astype(np.float64)
        ff = oracle_mod.ff_from_run_in(s.run_in, s.masses)
        o = oracle_mod.forces(ff, np.arange(1, s.n + 1), s.types, st["x"], st["v"], s.lo, Lb, 0)
        assert force_err(st["f"], o["f"]) < TOL, k
    b.run(5)
    b.close()


def test_tile_matches_list_schedule_over_steps():
    """Schedule 11 against the default schedule 8 over 20 steps from the same state: the
    same trajectory up to FP32 summation order."""
    from gpumdpd_b200 import Engine
    s = _systems()["melt_skin0"]
    a = _engine(s)
    b = Engine(s.run_in, system=s.c_system())
    b.set_tuning(pair_variant=8)
    a.run(20)
    b.run(20)
    sa, sb = a.state(), b.state()
    L = _box(a)
    dx = sa["x"] - sb["x"]
    dx -= L * np.round(dx / L)
    assert np.abs(dx).max() < 1e-3
    assert force_err(sa["f"], sb["f"]) < 1e-3
    ta, tb = a.thermo(), b.thermo()
    assert ta["temp"][-1] == pytest.approx(tb["temp"][-1], rel=1e-3)


@pytest.mark.parametrize("name", ["dpd_skin0", "dpd_skin03", "melt_skin0", "box3", "box4"])
def test_tile_list_build_matches_oracle(oracle_mod, name):
    """List-build variant 4 (the half list written from the tiles): the neighbour set equals
    the oracle's FP32-predicate set, and the list schedule's step-0 forces and the forces of
    the next 5 steps on the engine's own state are the oracle's."""
    from gpumdpd_b200 import Engine
    s = _systems()[name]
    s.run_in = re.sub(r"(?m)^thermo \d+$", "thermo 1000", s.run_in)
    e = Engine(s.run_in, system=s.c_system())
    e.set_tuning(pair_variant=8, build_variant=4)
    e.run(0)
    c = e.cells()
    got = e.neighbors()
    ref = oracle_mod.pairs_f32(np.arange(1, s.n + 1), c["cell"], c["offset"], c["nc"], c["w"], c["cut2"])
    assert len(got) == len(set(map(tuple, got.tolist())))
    assert set(map(tuple, got.tolist())) == set(map(tuple, ref.tolist()))
    ff = oracle_mod.ff_from_run_in(s.run_in, s.masses)
    tags = np.arange(1, s.n + 1)
    st = e.state()
    o = oracle_mod.forces(ff, tags, s.types, st["x"], st["v"], s.lo, _box(e), 0, bonds=s.bonds)
    assert force_err(st["f"], o["f"]) < TOL
    dt = float(re.search(r"(?m)^timestep (\S+)$", s.run_in).group(1))
    m = np.asarray(s.masses)[np.asarray(s.types) - 1][:, None]
    for k in range(1, 6):
        e.run(1)
        got = e.state()
        vh = got["v"] - 0.5 * dt * got["f"] / m
        o = oracle_mod.forces(ff, tags, s.types, got["x"], vh, s.lo, _box(e), k, bonds=s.bonds)
        assert force_err(got["f"], o["f"]) < TOL, k
    e.close()
