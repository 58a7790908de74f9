"""The FP64 oracle pinned against the reference's own outputs (golden fixtures made by
tests/golden/gen_ref_fixtures.py with the reference's CUDA build), CPU only."""
import numpy as np
import pytest

from conftest import force_err, load_golden

SYSTEMS = ["dpd_c1", "dpd_random_only", "mdpd_slab", "diblock", "mix_rc", "angle_chains", "wall_channel",
           "wall_reflect"]


def _state(g, step):
    x = np.column_stack([g[f"s{step}_{c}"] for c in "xyz"])
    v = np.column_stack([g[f"s{step}_v{c}"] for c in "xyz"])
    f = np.column_stack([g[f"s{step}_f{c}"] for c in "xyz"])
    return x, v, f, g[f"s{step}_id"], g[f"s{step}_type"]


def test_saru_bit_exact_against_reference(oracle_mod):
    """oracle_saru == the reference's saru (src/force/pair_dpd.cu:212-236), bit for bit."""
    g = dict(np.load(__import__("conftest").GOLDEN + "/ref_saru_kat.npz"))
    lib = oracle_mod.load()
    out = np.array([lib.oracle_saru(int(a), int(b), int(s), int(t))
                    for a, b, s, t in zip(g["t1"][:2000], g["t2"][:2000], g["seed"][:2000], g["step"][:2000])],
                   dtype=np.float32)
    assert np.array_equal(out.view(np.uint32), g["theta"][:2000].view(np.uint32))
    # the vectorised entry point over all records
    allout = np.array([lib.oracle_saru(int(a), int(b), int(s), int(t))
                       for a, b, s, t in zip(g["t1"], g["t2"], g["seed"], g["step"])], dtype=np.float32)
    assert np.array_equal(allout.view(np.uint32), g["theta"].view(np.uint32))
    # uniform on [-sqrt3, sqrt3] with unit variance
    assert abs(allout.mean()) < 0.03 and abs(allout.var() - 1.0) < 0.03
    assert allout.max() <= np.float32(1.7320508) and allout.min() >= -np.float32(1.7320508)


@pytest.mark.parametrize("name", SYSTEMS)
def test_step0_forces_match_reference(oracle_mod, name):
    """Oracle FP64 forces at step 0 from the reference's step-0 state vs the reference's
    FP32 forces (atomics; tolerance 1e-5 of the RMS force)."""
    g = load_golden(name)
    x, v, f_ref, ids, types = _state(g, 0)
    ff = oracle_mod.ff_from_run_in(str(g["run_in"]), g["masses"])
    L = g["hi"] - g["lo"]
    o = oracle_mod.forces(ff, ids, types, x, v, g["lo"], L, 0, bonds=g.get("bonds"), angles=g.get("angles"))
    assert force_err(o["f"], f_ref) < 1e-5


def test_step0_forces_match_reference_double_build(oracle_mod):
    """Against the reference's -DDOUBLE build the oracle agrees to the dump's print
    precision (%.9f): the only single-precision part left is Saru's float tail, which
    both evaluate identically."""
    g = load_golden("dpd_c1_double")
    x, v, f_ref, ids, types = _state(g, 0)
    ff = oracle_mod.ff_from_run_in(str(g["run_in"]), g["masses"])
    oracle_mod.set_saru_double_tail(True)
    try:
        o = oracle_mod.forces(ff, ids, types, x, v, g["lo"], g["hi"] - g["lo"], 0)
    finally:
        oracle_mod.set_saru_double_tail(False)
    assert np.abs(o["f"] - f_ref).max() < 5e-8


@pytest.mark.parametrize("name", SYSTEMS + ["dpd_c1_double"])
def test_step0_thermo_matches_reference(oracle_mod, name):
    """T, pair PE and the pressure tensor at step 0 (thermo.txt, src/compute/thermo.cu)."""
    g = load_golden(name)
    x, v, _, ids, types = _state(g, 0)
    ff = oracle_mod.ff_from_run_in(str(g["run_in"]), g["masses"])
    L = g["hi"] - g["lo"]
    o = oracle_mod.run(ff, ids, types, x, v, g["lo"], L, 1, 0, 1, bonds=g.get("bonds"), angles=g.get("angles"))
    th = o["thermo"]
    rtol = 2e-6 if name.endswith("double") else 2e-5
    assert th["temp"][0] == pytest.approx(g["thermo_temp"][0], rel=rtol, abs=2e-6)
    assert th["pair_pe"][0] == pytest.approx(g["thermo_pair_pe"][0], rel=rtol, abs=2e-6)
    assert th["pressure"][0] == pytest.approx(g["thermo_pressure"][0], rel=rtol, abs=2e-6)
    for k, c in enumerate(["pxx", "pxy", "pxz", "pyy", "pyz", "pzz"]):
        assert th[c][0] == pytest.approx(g[f"thermo_{c}"][0], rel=1e-4, abs=2e-5)
    if "thermo_bond_pe" in g:
        assert th["bond_pe"][0] == pytest.approx(g["thermo_bond_pe"][0], rel=rtol, abs=2e-6)
    if "thermo_angle_pe" in g:
        assert th["angle_pe"][0] == pytest.approx(g["thermo_angle_pe"][0], rel=rtol, abs=2e-6)


@pytest.mark.parametrize("name", ["dpd_c1", "mdpd_slab", "diblock", "dpd_c1_double", "angle_chains",
                                  "wall_channel", "wall_reflect"])
def test_trajectory_matches_reference(oracle_mod, name):
    """10 velocity-Verlet steps (src/main/utils.cuh:254-303) from the reference's step-0
    state: positions and forces at step 1 and 10 track the reference."""
    g = load_golden(name)
    x, v, _, ids, types = _state(g, 0)
    ff = oracle_mod.ff_from_run_in(str(g["run_in"]), g["masses"])
    L = g["hi"] - g["lo"]
    dbl = name.endswith("double")
    for steps in (1, 10):
        oracle_mod.set_saru_double_tail(dbl)
        try:
            o = oracle_mod.run(ff, ids, types, x, v, g["lo"], L, 1, steps, 1, bonds=g.get("bonds"),
                               angles=g.get("angles"))
        finally:
            oracle_mod.set_saru_double_tail(False)
        xr, vr, fr, _, _ = _state(g, steps)
        dx = o["x"] - xr
        dx -= L * np.round(dx / L)
        # the stiff angle term (float acos in the reference's build) makes its FP32
        # trajectory drift from the FP64 one about twice as fast over 10 steps
        slack = 4.0 if name == "angle_chains" and steps == 10 else 1.0
        tol_x = 1e-7 if dbl else (2e-6 if steps == 1 else 5e-5 * slack)
        assert np.abs(dx).max() < tol_x
        tol_f = 1e-7 if dbl else (2e-5 if steps == 1 else 3e-4 * slack)
        assert force_err(o["f"], fr) < tol_f
        # thermo rows of every step
        for k in range(steps + 1):
            assert o["thermo"]["temp"][k] == pytest.approx(g["thermo_temp"][k], rel=1e-4, abs=1e-5)


def test_oracle_conservation(oracle_mod):
    """Newton's third law (the reference's compute tf measures this) and zero net
    momentum change over a step for an isolated system."""
    g = load_golden("diblock")
    x, v, _, ids, types = _state(g, 0)
    ff = oracle_mod.ff_from_run_in(str(g["run_in"]), g["masses"])
    o = oracle_mod.forces(ff, ids, types, x, v, g["lo"], g["hi"] - g["lo"], 0, bonds=g["bonds"])
    assert np.abs(o["f"].sum(axis=0)).max() < 1e-9
    r = oracle_mod.run(ff, ids, types, x, v, g["lo"], g["hi"] - g["lo"], 1, 5, 1, bonds=g["bonds"])
    p0 = v.sum(axis=0)
    assert np.abs(r["v"].sum(axis=0) - p0).max() < 1e-9


def test_oracle_rdf_ideal_gas(oracle_mod):
    """g(r) of uniform random points is 1 within counting noise."""
    rng = np.random.default_rng(1)
    L = np.array([12.0, 12.0, 12.0])
    n = 5000
    x = rng.uniform(0, 12.0, (n, 3))
    types = np.where(np.arange(n) % 2 == 0, 1, 2).astype(np.int32)
    g = oracle_mod.rdf(types, x, [0, 0, 0], L, 1, 2, 3.0, 30)
    assert np.abs(g[10:] - 1.0).max() < 0.08
    g11 = oracle_mod.rdf(types, x, [0, 0, 0], L, 1, 1, 3.0, 30)
    assert np.abs(g11[10:] - 1.0).max() < 0.1


def test_oracle_pairs_f32_vs_f64(oracle_mod):
    """The FP32 cell-offset predicate selects the FP64 pair set except pairs within
    float rounding of the cutoff shell."""
    rng = np.random.default_rng(2)
    n, L, cut = 2000, 9.0, 1.3
    x = rng.uniform(0, L, (n, 3))
    nc = np.array([int(L // cut)] * 3, dtype=np.int32)
    w = np.float32(L / nc[0]) * np.ones(3, dtype=np.float32)
    cell = np.minimum((x // w.astype(np.float64)).astype(np.int32), nc - 1)
    off = (x - cell * w.astype(np.float64)).astype(np.float32)
    xe = cell * w.astype(np.float64) + off.astype(np.float64)
    Le = nc * w.astype(np.float64)
    tags = np.arange(1, n + 1)
    p32 = set(map(tuple, oracle_mod.pairs_f32(tags, cell, off, nc, w, np.float32(cut) * np.float32(cut)).tolist()))
    p64 = set(map(tuple, oracle_mod.pairs_f64(tags, xe, [0, 0, 0], Le, float(np.float32(cut))).tolist()))
    diff = p32 ^ p64
    assert len(diff) <= 2
    for a, b in diff:
        d = xe[a - 1] - xe[b - 1]
        d -= Le * np.round(d / Le)
        assert abs(np.linalg.norm(d) - float(np.float32(cut))) < 1e-5


def test_group_fixes_match_reference(oracle_mod):
    """fix spring (post_force, the zero step included), rvcm and recenter (end_of_step)
    over 10 steps from the reference's step-0 state: states after step 1, 3 (rvcm),
    4 (recenter) and 10, and the rows of the spring's record file (every 2 steps)."""
    g = load_golden("probe_fixes")
    x, v, f0, ids, types = _state(g, 0)
    ff = oracle_mod.ff_from_run_in(str(g["run_in"]), g["masses"])
    assert ff.spring_on and ff.rvcm_on and ff.recenter_on
    L = g["hi"] - g["lo"]
    m = g["masses"][types - 1]
    o0 = oracle_mod.forces(ff, ids, types, x, v, g["lo"], L, 0)
    # the dumped step-0 force includes the spring's share
    assert force_err(o0["f"], f0) > 1e-4
    z = oracle_mod.run(ff, ids, types, x, v, g["lo"], L, 1, 0, 1)
    assert force_err(z["f"], f0) < 1e-5
    for steps in (1, 3, 4, 10):
        o = oracle_mod.run(ff, ids, types, x, v, g["lo"], L, 1, steps, 1)
        xr, vr, fr, _, _ = _state(g, steps)
        dx = o["x"] - xr
        dx -= L * np.round(dx / L)
        assert np.abs(dx).max() < (2e-6 if steps == 1 else 5e-5), steps
        assert np.abs(o["v"] - vr).max() < (2e-5 if steps == 1 else 5e-4), steps
        assert force_err(o["f"], fr) < (2e-5 if steps == 1 else 3e-4), steps
        if steps == 3:  # rvcm with flags 1 0 1 at step 3: no x or z momentum left
            p_ref = (m[:, None] * vr).sum(0)
            p_o = (m[:, None] * o["v"]).sum(0)
            assert abs(p_ref[0]) < 1e-3 and abs(p_ref[2]) < 1e-3 and abs(p_ref[1]) > 1e-2
            assert abs(p_o[0]) < 1e-9 and abs(p_o[2]) < 1e-9
        if steps == 4:  # recenter at step 4: the probe's centre of mass is at the target
            grp = types == 2
            com = (m[grp, None] * (o["x"] + o["image"] * L)[grp]).sum(0) / m[grp].sum()
            np.testing.assert_allclose(com, list(ff.recenter_c), atol=1e-9)
    rows = g["spring"]
    assert list(rows[:, 0]) == [0, 2, 4, 6, 8, 10]
    for row in rows:
        # the spring of step s acts before that step's end_of_step fixes (a recenter at
        # step 4 or 8 comes after the record)
        oracle_mod.run(ff, ids, types, x, v, g["lo"], L, 1, int(row[0]), 1)
        want = oracle_mod.spring_last()
        np.testing.assert_allclose(row[1:], want, rtol=2e-4, atol=2e-4 * np.abs(want[:4]).max())
