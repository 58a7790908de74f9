"""The autotuner: it times every candidate (skin = cell size, safe rebuild check interval,
pair schedule, tile edge, launch mode, cell order with its list build) over whole steps and returns the fastest; every
candidate it may return is a valid configuration of the same system (its step-0 forces
are the FP64 oracle's within 1e-5 of the RMS force)."""
import numpy as np
import pytest

from conftest import force_err

pytestmark = pytest.mark.gpu


def test_tune_system_picks_the_fastest_exact_candidate(oracle_mod):
    from gpumdpd_b200 import Engine, inputs, tune
    s = inputs.plain_dpd(L=8.0, seed=3, nsteps=100)
    schedules = ({"pair_variant": 8}, {"pair_variant": 11, "tile": 0}, {"pair_variant": 11, "tile": 2})
    best, table = tune.tune_system(s, skins=(0.0, 0.3), schedules=schedules, launch_modes=(0, 1),
                                   intervals=(1, 2, 5), steps=5, warmup=2)
    timed = [t for t in table if "ms_per_step" in t]
    assert best["ms_per_step"] == min(t["ms_per_step"] for t in timed)
    assert all(t["ms_per_step"] > 0 for t in timed)
    assert {t["skin"] for t in timed} == {0.0, 0.3}
    assert {t["launch_mode"] for t in timed} == {0, 1}
    assert {(t["pair_variant"], t.get("tile")) for t in timed} == {(8, None), (11, 0), (11, 2)}
    assert {(t["cell_order"], t["build_variant"]) for t in timed} == {(0, 5), (1, 0)}
    assert all(t["nl_f"] == 1 for t in timed if t["skin"] == 0.0)
    ff = oracle_mod.ff_from_run_in(s.run_in, s.masses)
    for t in timed:
        knobs = {k: t[k] for k in ("pair_variant", "launch_mode", "tile", "cell_order", "build_variant") if k in t}
        e = Engine(tune.with_skin(s.run_in, t["skin"], t["nl_f"]), system=s.c_system())
        e.set_tuning(**knobs)
        e.run(0)
        st = e.state()
        c = e.cells()
        L = c["nc"].astype(np.float64) * c["w"].astype(np.float64)
        o = oracle_mod.forces(ff, np.arange(1, s.n + 1), s.types, st["x"], st["v"], s.lo, L, 0)
        assert force_err(st["f"], o["f"]) < 1e-5, t
        e.close()


def test_tune_batch_and_too_small_boxes():
    from gpumdpd_b200 import inputs, tune
    systems = [inputs.binary_mixture(L, 30.0, seed=k) for k, L in enumerate((4.5, 6.0, 8.0))]
    best, table = tune.tune_batch(systems, skins=(0.0, 0.3), variants=(8, 11), launch_modes=(0,), steps=3,
                                  warmup=1)
    # a 4.5 box holds 3 cells of 1.3 at skin 0.3 but 4 at skin 0: both are valid
    assert {t["skin"] for t in table} == {0.0, 0.3}
    assert "ms_per_step" in best
    tiny = inputs.binary_mixture(3.5, 30.0, seed=9)   # fewer than 3 cells at skin 0.3
    best, table = tune.tune_system(tiny, skins=(0.0, 0.3), variants=(8,), launch_modes=(0,), steps=3, warmup=1)
    assert any("error" in t for t in table) and best["skin"] == 0.0
