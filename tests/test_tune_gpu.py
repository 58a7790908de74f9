"""The autotuner: it times each candidate skin x pair schedule over whole steps and returns
the fastest; every candidate it may return is a valid configuration of the same system."""
import pytest

pytestmark = pytest.mark.gpu


def test_tune_system_picks_a_timed_candidate():
    from gpumdpd_b200 import inputs, tune
    s = inputs.plain_dpd(L=8.0, seed=3, nsteps=100)
    best, table = tune.tune_system(s, skins=(0.0, 0.3), variants=(1, 8), steps=5, warmup=2)
    timed = [t for t in table if "ms_per_step" in t]
    assert len(timed) == 4
    assert best["ms_per_step"] == min(t["ms_per_step"] for t in timed)
    assert all(t["ms_per_step"] > 0 for t in timed)


def test_tune_batch_and_too_small_boxes():
    from gpumdpd_b200 import inputs, tune
    systems = [inputs.binary_mixture(L, 30.0, seed=k) for k, L in enumerate((4.5, 6.0, 8.0))]
    best, table = tune.tune_batch(systems, skins=(0.0, 0.3), variants=(8,), steps=3, warmup=1)
    # a 4.5 box holds 3 cells of 1.3 at skin 0.3 but 4 at skin 0: both are valid
    assert {t["skin"] for t in table} == {0.0, 0.3}
    assert "ms_per_step" in best
    tiny = inputs.binary_mixture(3.5, 30.0, seed=9)   # fewer than 3 cells at skin 0.3
    best, table = tune.tune_system(tiny, skins=(0.0, 0.3), variants=(8,), steps=3, warmup=1)
    assert any("error" in t for t in table) and best["skin"] == 0.0
