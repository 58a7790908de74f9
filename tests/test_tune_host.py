"""Host logic of the autotuner (no GPU): the run.in rewrite of the `neighbor` command and
the rule that keeps only rebuild check intervals that cannot miss a rebuild, the candidate
table, and the tuning struct the knobs fill."""
import pytest

from gpumdpd_b200 import inputs, tune


def test_with_skin_and_interval():
    s = inputs.plain_dpd(L=8.0, seed=3, nsteps=100)
    t = tune.with_skin(s.run_in, 0.2, 5)
    line = [ln for ln in t.splitlines() if ln.startswith("neighbor")][0].split()
    assert float(line[2]) == 0.2 and line[4] == "5"
    t = tune.with_skin(s.run_in, 0.1)
    line2 = [ln for ln in t.splitlines() if ln.startswith("neighbor")][0].split()
    assert float(line2[2]) == 0.1 and line2[4] == [ln for ln in s.run_in.splitlines()
                                                   if ln.startswith("neighbor")][0].split()[4]


def test_safe_intervals():
    # skin 0: the list is rebuilt every step whatever the interval
    assert tune.safe_intervals(0.0, 0.1) == (1,)
    # skin 0.3, largest step 0.04: 1.5 * k * 0.04 < 0.15 for k = 1, 2 only
    assert tune.safe_intervals(0.3, 0.04, (1, 2, 5)) == (1, 2)
    # a fast particle (0.2 per step) leaves only the check every step
    assert tune.safe_intervals(0.3, 0.2, (1, 2, 5)) == (1,)
    assert tune.safe_intervals(1.0, 0.01, (1, 2, 5, 10)) == (1, 2, 5, 10)


def test_candidates_cover_every_knob_combination():
    from gpumdpd_b200 import tune
    sc = ({"pair_variant": 8}, {"pair_variant": 11, "tile": 2})
    got = list(tune._candidates(sc, (0, 1), tune.LISTS))
    assert len(got) == 2 * 2 * len(tune.LISTS)
    assert {(c["pair_variant"], c["launch_mode"], c["cell_order"], c["build_variant"]) for c in got} == \
        {(p, m, o, b) for p in (8, 11) for m in (0, 1) for o, b in ((0, 5), (1, 0))}
    assert all(c["tile"] == 2 for c in got if c["pair_variant"] == 11)


def test_tuning_struct_defaults_and_overrides():
    from gpumdpd_b200 import capi
    t = capi.tuning()
    assert (t.pair_variant, t.cell_order, t.build_variant, t.launch_mode) == (8, 0, 5, 0)
    t = capi.tuning(cell_order=1, build_variant=0, launch_mode=3)
    assert (t.pair_variant, t.cell_order, t.build_variant, t.launch_mode) == (8, 1, 0, 3)
    with pytest.raises(TypeError):
        capi.tuning(no_such_knob=1)
