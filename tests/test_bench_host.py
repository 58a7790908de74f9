"""Host helpers of bench.py (no GPU): the thermo cadence shared by both arms, the run.in
rewrites of the FP64 comparison windows, the block-averaged statistics and the rounding of
the printed line."""
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


class _Args:
    def __init__(self, warmup, steps):
        self.warmup, self.steps = warmup, steps


def test_thermo_cadence_divides_warmup_and_steps():
    import bench
    for w, k in ((5, 20), (5, 1000), (3, 1000), (10, 200), (4, 6)):
        g = bench.thermo_every(_Args(w, k))
        assert w % g == 0 and k % g == 0
        assert g == math.gcd(w, k)


def test_run_in_rewrites():
    import bench
    from gpumdpd_b200 import inputs
    s = inputs.binary_mixture(6.0, 30.0, seed=1, nsteps=77, thermo=9, rdf=(2.0, 50, 10))
    assert "compute " in s.run_in
    t = bench.with_run(bench.with_thermo(bench.without_computes(s.run_in), 5), 300)
    lines = t.splitlines()
    assert "thermo 5" in lines and "run 300" in lines
    assert not any(ln.startswith("compute ") for ln in lines)
    # everything else is kept
    assert [ln for ln in lines if ln.startswith(("pair_", "neighbor", "timestep", "fix", "group"))] == \
        [ln for ln in s.run_in.splitlines() if ln.startswith(("pair_", "neighbor", "timestep", "fix", "group"))]


def test_block_stats_and_compare():
    import bench
    rng = np.random.default_rng(3)
    x = rng.normal(2.0, 0.5, 4000)
    m, se = bench.block_stats(x, 10)
    assert m == pytest.approx(x.mean())
    assert se == pytest.approx(0.5 / math.sqrt(4000), rel=0.5)  # uncorrelated samples
    # two blocks of at least two rows are needed for an error estimate
    assert not math.isnan(bench.block_stats([1.0, 2.0, 3.0, 4.0], 10)[1])
    assert math.isnan(bench.block_stats([1.0, 2.0, 3.0], 10)[1])
    c = bench.compare(x + 0.01, x)
    assert set(c) == {"fp32", "fp64", "err", "stderr", "z"}
    assert c["err"] == pytest.approx(0.01, abs=1e-6)


def test_compact_rounds_floats_only():
    import bench
    d = {"a": 3224569365.9103823, "b": [0.000123456789, 7], "c": {"d": "text", "e": float("nan")}, "f": 12}
    c = bench.compact(d)
    assert c["a"] == 3.225e9 and c["b"] == [0.0001235, 7] and c["c"]["d"] == "text"
    assert c["c"]["e"] is None and c["f"] == 12
