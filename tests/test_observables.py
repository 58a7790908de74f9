"""Slab observables (density profile, surface tension) and the tuner's input rewrite,
on synthetic data with known answers (CPU)."""
import numpy as np
import pytest

from gpumdpd_b200 import inputs, observables, tune


def test_density_profile_of_a_uniform_slab():
    s = inputs.mdpd_slab(Lx=10.0, Ly=10.0, Lz=30.0, z0=10.0, z1=20.0, rho=6.0, seed=3, nsteps=10)
    c, rho = observables.density_profile(s.x, s.lo, s.hi, axis=2, width=0.5)
    assert len(c) == 60
    assert rho.sum() * 0.5 * 100.0 == pytest.approx(s.n)
    liq, vap = observables.slab_densities(c, rho, 10.0, 20.0, margin=1.0)
    assert liq == pytest.approx(6.0, rel=0.05)
    assert vap == 0.0


def test_surface_tension_formula():
    rng = np.random.default_rng(0)
    p = np.zeros((4000, 6))
    p[:, 0] = 2.0 + 0.1 * rng.normal(size=4000)   # pxx
    p[:, 3] = 2.0 + 0.1 * rng.normal(size=4000)   # pyy
    p[:, 5] = 3.0 + 0.1 * rng.normal(size=4000)   # pzz
    g, err = observables.surface_tension(p, Lz=120.0)
    assert g == pytest.approx(60.0, abs=5 * err)
    assert 0 < err < 1.0


def test_with_skin_rewrites_only_the_skin():
    s = inputs.plain_dpd(L=8.0, seed=1, nsteps=10, skin=0.3)
    t = tune.with_skin(s.run_in, 0.1)
    line = [ln for ln in t.splitlines() if ln.startswith("neighbor")][0]
    assert line.split()[1:] == ["1.0", "0.1", "10.0", "1"]
    assert t.replace(line, "") == s.run_in.replace(
        [ln for ln in s.run_in.splitlines() if ln.startswith("neighbor")][0], "")
