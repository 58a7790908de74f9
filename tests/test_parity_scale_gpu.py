"""Parity on the headline configurations at full size, through the C ABI.

- The A5B5 diblock melt (L = 100, N = 3.0M, 2.7M harmonic bonds, skin 0: the
  configuration the headline throughput is measured on) under the default knobs (linear
  cell order, column-range list build), the column cell order, and the Morton cell order
  with the cell-by-cell build: step-0 forces within 1e-5 of the RMS force against the FP64 oracle on the engine's own
  state, and the neighbour set equal to the oracle's FP32-predicate set
  (src/force/neigh_list.cu:360-389) as tag pairs.
- The packed 256-replica A/B sweep (3.16M slots, L log-uniform over 8..24, a_AB over
  25..45, skin 0): for 8 replicas (smallest, largest, a_AB extremes and four between),
  step-0 forces and the forces of each of steps 1-10 on the engine's own state within
  1e-5 of the RMS force.
"""
import re

import numpy as np
import pytest

from conftest import force_err

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def _pair_keys(p):
    p = np.asarray(p, dtype=np.int64)
    a, b = np.minimum(p[:, 0], p[:, 1]), np.maximum(p[:, 0], p[:, 1])
    return np.sort(a << 32 | b)


def _engine_box(s, cut=1.0):
    """The engine's periodic box: nc cells of the float cell width w = (float)(L / nc),
    nc = floor(L / (global_cut + skin)) per dimension."""
    L = np.asarray(s.box, dtype=np.float64)
    nc = np.floor(L / cut)
    return nc * (L / nc).astype(np.float32).astype(np.float64)


def _half_v(st, masses, types, dt):
    m = np.asarray(masses)[np.asarray(types) - 1][:, None]
    return st["v"] - 0.5 * dt * st["f"] / m


@pytest.mark.parametrize("tuning", [{}, {"cell_order": 2}, {"cell_order": 1, "build_variant": 0}],
                         ids=["linear_columns", "columns", "morton"])
def test_melt_3M_step0_forces_and_neighbor_set(oracle_mod, tuning):
    from gpumdpd_b200 import Engine, inputs
    s = inputs.diblock_melt(L=100.0, seed=7, nsteps=10, thermo=1000, skin=0.0)
    assert s.n == 3_000_000
    e = Engine(s.run_in, system=s.c_system())
    e.set_tuning(pair_variant=8, **tuning)
    e.run(0)
    st = e.state()
    c = e.cells()
    L = c["nc"].astype(np.float64) * c["w"].astype(np.float64)
    ff = oracle_mod.ff_from_run_in(s.run_in, s.masses)
    tags = np.arange(1, s.n + 1)
    o = oracle_mod.forces(ff, tags, s.types, st["x"], st["v"], s.lo, L, 0, bonds=s.bonds)
    assert force_err(st["f"], o["f"]) < FORCE_TOL
    th = e.thermo()
    assert th["pair_pe"][0] == pytest.approx(o["pair_pe"], rel=1e-6)
    assert th["bond_pe"][0] == pytest.approx(o["bond_pe"], rel=1e-6)
    got = e.neighbors()
    ref = oracle_mod.pairs_f32(tags, c["cell"], c["offset"], c["nc"], c["w"], c["cut2"])
    assert len(got) == len(ref)
    kg = _pair_keys(got)
    assert np.all(kg[1:] != kg[:-1])  # no duplicates
    assert np.array_equal(kg, _pair_keys(ref))
    e.close()


def test_packed_sweep_replicas_every_step(oracle_mod):
    from gpumdpd_b200 import Batch, inputs, tune
    systems = inputs.replica_sweep(n_rep=256, nsteps=5000, thermo=10)
    for s in systems:
        s.run_in = tune.with_skin(s.run_in, 0.0)
    b = Batch([s.run_in for s in systems], [s.c_system() for s in systems],
              tuning={"pair_variant": 8})
    assert sum(s.n for s in systems) > 3_000_000
    ns = np.array([s.n for s in systems])
    sel = sorted({int(np.argmin(ns)), int(np.argmax(ns)), 0, 255} | {int(k) for k in np.linspace(0, 255, 6)[1:-1]})
    ffs = {k: oracle_mod.ff_from_run_in(systems[k].run_in, systems[k].masses) for k in sel}
    b.run(0)
    for k in sel:
        s = systems[k]
        st = b.state(k)
        o = oracle_mod.forces(ffs[k], np.arange(1, s.n + 1), s.types, st["x"], st["v"], s.lo, _engine_box(s), 0)
        assert force_err(st["f"], o["f"]) < FORCE_TOL, (k, 0)
    dt = float(re.search(r"(?m)^timestep (\S+)$", systems[0].run_in).group(1))
    for step in range(1, 11):
        b.run(1)
        for k in sel:
            s = systems[k]
            st = b.state(k)
            o = oracle_mod.forces(ffs[k], np.arange(1, s.n + 1), s.types, st["x"],
                                  _half_v(st, s.masses, s.types, dt), s.lo, _engine_box(s), step)
            assert force_err(st["f"], o["f"]) < FORCE_TOL, (k, step)
    b.close()
