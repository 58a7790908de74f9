"""The FP64 parity engine (dpd_create_fp64; Engine(..., precision="fp64")) against the
reference's -DDOUBLE build and the FP64 oracle.

Stated tolerances: against the -DDOUBLE build's golden dump (printed with %.9f) step-0
forces within 5e-8 and positions/forces after 1 and 10 steps within 1e-7, thermo rows
within its print precision; against the FP64 oracle (Saru tail of the -DDOUBLE build)
positions within 1e-9 and forces within 1e-9 of the RMS force after 10 steps, thermo rows
within 1e-9 relative: only FP64 summation order separates the two.  The single-precision
engine meets 1e-5 on the same comparisons."""
import numpy as np
import pytest

from conftest import force_err, load_golden

pytestmark = pytest.mark.gpu


def _golden_system(name):
    from gpumdpd_b200.inputs import System
    g = load_golden(name)
    x = np.column_stack([g[f"s0_{c}"] for c in "xyz"])
    v = np.column_stack([g[f"s0_v{c}"] for c in "xyz"])
    run_in = str(g["run_in"])
    style = "angle" if "angles" in g else ("bond" if "bonds" in g else "atomic")
    lines = [ln for ln in run_in.splitlines() if not ln.startswith("dump")]
    s = System(g["lo"], g["hi"], g["masses"], g["s0_type"], x, v, bonds=g.get("bonds"),
               n_bondtypes=1 if "bonds" in g else 0, run_in="\n".join(lines) + "\n", atom_style=style,
               angles=g.get("angles"), n_angletypes=1 if "angles" in g else 0)
    return s, g


def _golden_state(g, step):
    x = np.column_stack([g[f"s{step}_{c}"] for c in "xyz"])
    f = np.column_stack([g[f"s{step}_f{c}"] for c in "xyz"])
    order = np.argsort(g[f"s{step}_id"])
    return x[order], f[order]


def _fp64(system):
    from gpumdpd_b200 import Engine
    return Engine(system.run_in, system=system.c_system(), precision="fp64")


def test_fp64_engine_tracks_reference_double_build():
    """C1 (3000 particles) from the -DDOUBLE build's own step-0 state: forces at step 0, the
    state after 1 and 10 velocity-Verlet steps, and the 11 thermo rows."""
    s, g = _golden_system("dpd_c1_double")
    e = _fp64(s)
    e.run(0)
    x0, f0 = _golden_state(g, 0)
    st = e.state()
    assert np.abs(st["f"] - f0).max() < 5e-8
    L = s.hi - s.lo
    done = 0
    for steps in (1, 10):
        e.run(steps - done)
        done = steps
        xr, fr = _golden_state(g, steps)
        st = e.state()
        dx = st["x"] - xr
        dx -= L * np.round(dx / L)
        assert np.abs(dx).max() < 1e-7
        assert np.abs(st["f"] - fr).max() < 1e-7
    th = e.thermo()
    np.testing.assert_array_equal(th["step"], g["thermo_step"].astype(np.int64))
    for k in ("temp", "pair_pe", "pressure", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz"):
        ours = th[k] if k in th else th["p"][:, ["pxx", "pxy", "pxz", "pyy", "pyz", "pzz"].index(k)]
        np.testing.assert_allclose(ours, g[f"thermo_{k}"], rtol=0, atol=1.5e-6)


@pytest.mark.parametrize("name", ["mdpd_slab", "diblock", "mix_rc", "angle_chains", "dpd_random_only"])
def test_fp64_engine_matches_fp64_oracle(oracle_mod, name):
    """Ten steps of DPD, mDPD, bonded chains, per-pair cutoffs and angles against the FP64
    oracle with the -DDOUBLE build's Saru tail: agreement to FP64 summation order."""
    s, g = _golden_system(name)
    e = _fp64(s)
    e.run(10)
    st = e.state()
    ff = oracle_mod.ff_from_run_in(s.run_in, s.masses)
    L = s.hi - s.lo
    oracle_mod.set_saru_double_tail(True)
    try:
        o = oracle_mod.run(ff, np.arange(1, s.n + 1), s.types, s.x, s.v, s.lo, L, 1, 10, 1,
                           bonds=s.bonds, angles=s.angles)
    finally:
        oracle_mod.set_saru_double_tail(False)
    dx = st["x"] - o["x"]
    dx -= L * np.round(dx / L)
    assert np.abs(dx).max() < 1e-9
    assert np.abs(st["v"] - o["v"]).max() < 1e-9
    assert force_err(st["f"], o["f"]) < 1e-9
    th = e.thermo()
    assert len(th["step"]) == 11
    for k in ("temp", "pair_pe", "bond_pe", "angle_pe", "pressure"):
        np.testing.assert_allclose(th[k], o["thermo"][k], rtol=1e-9, atol=1e-9)


def test_fp64_engine_repeats_bit_for_bit():
    """No force atomics and fixed summation orders: two runs give identical states."""
    from gpumdpd_b200 import inputs
    s = inputs.diblock_melt(L=8.0, seed=52, nsteps=50, thermo=5)
    out = []
    for _ in range(2):
        e = _fp64(s)
        e.run(30)
        out.append((e.state(), e.thermo()))
    for k in ("x", "v", "f", "image"):
        np.testing.assert_array_equal(out[0][0][k], out[1][0][k])
    np.testing.assert_array_equal(out[0][1]["pressure"], out[1][1]["pressure"])


def test_fp64_engine_against_fp32_engine():
    """The FP32 engine and the FP64 engine from the same state: step-0 forces agree to the
    FP32 engine's precision, and the step counters, rows and set_state semantics match."""
    from gpumdpd_b200 import Engine, inputs
    s = inputs.plain_dpd(L=10.0, seed=2024, nsteps=20, thermo=5)
    a = Engine(s.run_in, system=s.c_system())
    b = _fp64(s)
    a.run(0)
    b.run(0)
    sa, sb = a.state(), b.state()
    assert force_err(sa["f"], sb["f"]) < 1e-5
    a.run(20)
    b.run(20)
    ta, tb = a.thermo(), b.thermo()
    np.testing.assert_array_equal(ta["step"], tb["step"])
    assert a.info()["step"] == b.info()["step"] == 20
    # set_state: the next run starts with a zero step at the current step counter
    st = b.state()
    a.set_state(st["x"], st["v"])
    b.set_state(st["x"], st["v"])
    a.run(5)
    b.run(5)
    assert a.info()["step"] == b.info()["step"]
    np.testing.assert_array_equal(a.thermo()["step"], b.thermo()["step"])


def test_fp64_handle_refuses_other_calls():
    from gpumdpd_b200 import DpdError, inputs
    s = inputs.plain_dpd(L=8.0, seed=3, nsteps=10)
    e = _fp64(s)
    with pytest.raises(DpdError) as ex:
        e.neighbors()
    assert "FP64 parity mode" in str(ex.value)
    e.run(2)
    assert e.info()["step"] == 2


def test_fp64_fene_bonds_match_fp64_oracle(oracle_mod):
    """FENE + WCA bonds (not in the reference): step-0 forces and bond PE, then ten steps,
    against the FP64 oracle.  Bonds start at 0.9 with the WCA range 2^(1/6) 0.85 = 0.954, so
    the repulsion acts.  The stiff FENE spring needs a shorter step than DPD's 0.04: with it,
    bonds pass R0 within ten steps, an error in both."""
    from gpumdpd_b200 import inputs
    s = inputs.diblock_melt(L=10.0, seed=9, nsteps=10, bond_step=0.9, thermo=1, dt=0.005)
    s.run_in = s.run_in.replace("bond_style harmonic", "bond_style fene").replace(
        "bond_coeff 1 4.0 0.0", "bond_coeff 1 30.0 1.5 1.0 0.85")
    assert "bond_style fene" in s.run_in and "bond_coeff 1 30.0 1.5 1.0 0.85" in s.run_in
    e = _fp64(s)
    e.run(0)
    st = e.state()
    ff = oracle_mod.ff_from_run_in(s.run_in, s.masses)
    L = s.hi - s.lo
    oracle_mod.set_saru_double_tail(True)
    try:
        o0 = oracle_mod.forces(ff, np.arange(1, s.n + 1), s.types, s.x, s.v, s.lo, L, 0, bonds=s.bonds)
        o = oracle_mod.run(ff, np.arange(1, s.n + 1), s.types, s.x, s.v, s.lo, L, 1, 10, 1, bonds=s.bonds)
    finally:
        oracle_mod.set_saru_double_tail(False)
    assert force_err(st["f"], o0["f"]) < 1e-12
    assert e.thermo()["bond_pe"][0] == pytest.approx(o0["bond_pe"], rel=1e-12)
    e.run(10)
    st = e.state()
    dx = st["x"] - o["x"]
    dx -= L * np.round(dx / L)
    assert np.abs(dx).max() < 1e-9
    assert force_err(st["f"], o["f"]) < 1e-9
    np.testing.assert_allclose(e.thermo()["bond_pe"], o["thermo"]["bond_pe"], rtol=1e-9)
