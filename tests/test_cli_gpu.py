"""The gpudpd_b200 executable against the reference's own executable on the same run.in and
data file: thermo.txt, the all.trj frames of a `dump` command, the record file of a
`fix spring` and the data file of `write_data`.

Stated tolerances: step-0 values agree to the reference's FP32 precision (positions 1e-6,
forces 1e-5 of the RMS force, thermo 2e-5 relative); later frames within the FP32
trajectory tolerances of the 10-step parity tests (positions 5e-5 after 10 steps)."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "gpumdpd_b200", "gpudpd_b200")
STOCK = os.path.join(ROOT, "oracle", "_ref", "gpudpd_single")


def parse_trj(path):
    frames = {}
    lines = open(path).read().splitlines()
    k = 0
    while k < len(lines):
        assert lines[k] == "ITEM: TIMESTEP"
        step = int(lines[k + 1])
        assert lines[k + 2] == "ITEM: NUMBER OF ATOMS"
        n = int(lines[k + 3])
        assert lines[k + 4] == "ITEM: BOX BOUNDS pp pp pp"
        box = np.array([[float(v) for v in lines[k + 5 + q].split()] for q in range(3)])
        cols = lines[k + 8].split()[2:]
        data = np.array([[float(v) for v in ln.split()] for ln in lines[k + 9: k + 9 + n]])
        frames[step] = {"box": box, "cols": cols, **{c: data[:, q] for q, c in enumerate(cols)}}
        k += 9 + n
    return frames


def _run(binary, system, run_in, files, args=()):
    with tempfile.TemporaryDirectory() as td:
        open(os.path.join(td, "run.in"), "w").write(run_in)
        system.write_data(os.path.join(td, "system.data"))
        p = subprocess.run([binary, *args], cwd=td, capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
        return {f: open(os.path.join(td, f)).read() for f in files if os.path.exists(os.path.join(td, f))}


def _thermo(text):
    lines = [ln for ln in text.split("\n") if ln.strip()]
    head = lines[0].split()
    rows = np.array([[float(v) for v in ln.split()] for ln in lines[1:]])
    return head, {k: rows[:, i] for i, k in enumerate(head)}


def _case(wrapped):
    from gpumdpd_b200 import inputs
    s = inputs.probe_fixes(L=9.0, seed=41, nsteps=10, thermo=1)
    run_in = re.sub(r"(?m)^read_data .*$", "read_data system.data", s.run_in)
    run_in += f"dump 0 5 {'wrapped' if wrapped else 'unwrapped'} force_yes vel_yes\nwrite_data out.data\n"
    run_in += ("compute ct probe temp 2 temp.txt\ncompute cr all rho 1 0.0 4.5 0.0 9.0 2.0 7.0 rho.txt\n"
               "compute cm all msd 5 msd.txt\ncompute cf probe tf 1 tf.txt\n")
    return s, run_in


COMPUTE_FILES = {"temp.txt": [0, 2, 4, 6, 8, 10], "rho.txt": list(range(11)), "msd.txt": [0, 5, 10],
                 "tf.txt": list(range(11))}


@pytest.mark.skipif(not os.path.exists(CLI), reason="gpudpd_b200 not built")
@pytest.mark.parametrize("wrapped", [True, False])
def test_cli_outputs_match_reference_executable(wrapped):
    s, run_in = _case(wrapped)
    files = ["thermo.txt", "all.trj", "spring.txt", "out.data"] + list(COMPUTE_FILES)
    ours = _run(CLI, s, run_in, files)
    assert set(ours) == set(files)
    fr = parse_trj_text(ours["all.trj"])
    assert sorted(fr) == [0, 5, 10]
    for st, f in fr.items():
        assert f["cols"] == ["id", "type", "x", "y", "z", "fx", "fy", "fz", "vx", "vy", "vz"]
        np.testing.assert_array_equal(f["id"], np.arange(1, s.n + 1))
        np.testing.assert_array_equal(f["type"], s.types)
        np.testing.assert_allclose(f["box"], np.column_stack([s.lo, s.hi]))
    x0 = np.column_stack([fr[0][c] for c in "xyz"])
    np.testing.assert_allclose(x0, s.x, atol=2e-6)
    head, th = _thermo(ours["thermo.txt"])
    assert list(th["step"]) == list(range(11))
    spring = np.loadtxt(ours["spring.txt"].splitlines()[1:], ndmin=2)
    assert list(spring[:, 0]) == [0, 2, 4, 6, 8, 10]
    assert "Atoms" in ours["out.data"] and "Velocities" in ours["out.data"]
    comp = {f: _thermo(ours[f]) for f in COMPUTE_FILES}
    for f, steps in COMPUTE_FILES.items():
        assert list(comp[f][1]["step"]) == steps, f
    assert comp["tf.txt"][0] == ["step", "tf_x", "tf_y", "tf_z"]
    assert comp["msd.txt"][1]["msd"][0] < 1e-10
    if not os.path.exists(STOCK):
        pytest.skip("reference build (oracle/build_ref.sh SINGLE) not present")
    ref = _run(STOCK, s, run_in, files)
    rhead, rth = _thermo(ref["thermo.txt"])
    assert head == rhead
    for k in ("temp", "pair_pe", "pressure"):
        assert th[k][0] == pytest.approx(rth[k][0], rel=2e-5, abs=2e-6)
        np.testing.assert_allclose(th[k], rth[k], rtol=2e-3, atol=2e-3)
    rfr = parse_trj_text(ref["all.trj"])
    assert sorted(rfr) == sorted(fr)
    for st in fr:
        assert rfr[st]["cols"] == fr[st]["cols"]
        d = np.column_stack([fr[st][c] - rfr[st][c] for c in "xyz"])
        if wrapped:
            d -= (s.hi - s.lo) * np.round(d / (s.hi - s.lo))
        assert np.abs(d).max() < (2e-6 if st == 0 else 5e-5), st
        f = np.column_stack([fr[st]["f" + c] for c in "xyz"])
        rf = np.column_stack([rfr[st]["f" + c] for c in "xyz"])
        rms = np.sqrt((rf ** 2).sum(1).mean())
        assert np.linalg.norm(f - rf, axis=1).max() / rms < (1e-5 if st == 0 else 3e-4), st
        v = np.column_stack([fr[st]["v" + c] for c in "xyz"])
        rv = np.column_stack([rfr[st]["v" + c] for c in "xyz"])
        assert np.abs(v - rv).max() < (1e-6 if st == 0 else 5e-4), st
    # group computes: same headers and steps; step-0 values to FP32 precision (the rho count
    # may differ by a particle sitting on a region face), later rows within the trajectory
    # tolerance
    for f in COMPUTE_FILES:
        h, c = comp[f]
        rh, rc = _thermo(ref[f])
        assert h == rh, f
        np.testing.assert_array_equal(c["step"], rc["step"])
    vol = 4.5 * 9.0 * 5.0
    assert np.abs(comp["rho.txt"][1]["rho"] - _thermo(ref["rho.txt"])[1]["rho"]).max() * vol <= 1.5
    t, rt = comp["temp.txt"][1]["temp"], _thermo(ref["temp.txt"])[1]["temp"]
    assert t[0] == pytest.approx(rt[0], rel=1e-5)
    np.testing.assert_allclose(t, rt, rtol=1e-3)
    msd, rmsd = comp["msd.txt"][1]["msd"], _thermo(ref["msd.txt"])[1]["msd"]
    np.testing.assert_allclose(msd, rmsd, rtol=1e-3, atol=1e-6)
    tfc, rtf = comp["tf.txt"][1], _thermo(ref["tf.txt"])[1]
    fscale = np.abs(np.column_stack([fr[0]["f" + c] for c in "xyz"])).max()
    for c in ("tf_x", "tf_y", "tf_z"):
        assert abs(tfc[c][0] - rtf[c][0]) < 1e-4 * fscale
        np.testing.assert_allclose(tfc[c], rtf[c], atol=2e-2 * fscale)
    rspring = np.loadtxt(ref["spring.txt"].splitlines()[1:], ndmin=2)
    np.testing.assert_array_equal(spring[:, 0], rspring[:, 0])
    np.testing.assert_allclose(spring[:, 1:], rspring[:, 1:], rtol=2e-4, atol=2e-4 * np.abs(rspring[:, 1:5]).max())


def parse_trj_text(text):
    with tempfile.NamedTemporaryFile("w", suffix=".trj", delete=False) as f:
        f.write(text)
    try:
        return parse_trj(f.name)
    finally:
        os.unlink(f.name)


def test_engine_dump_frames_match_states(tmp_path):
    """Frames written during one run (snapshots taken while the device keeps stepping)
    equal the states of the same steps read between split runs, and the dump does not
    change the trajectory."""
    from gpumdpd_b200 import Engine, inputs
    s = inputs.binary_mixture(8.0, 35.0, seed=12, nsteps=12, thermo=4)
    path = tmp_path / "t.trj"
    e = Engine(s.run_in, system=s.c_system())
    e.dump_open(path, start=2, every=4, unwrapped=True, force=True, vel=True)
    e.run(0)
    e.run(12)
    e.dump_close()
    fr = parse_trj(str(path))
    assert sorted(fr) == [2, 6, 10]
    ref = Engine(s.run_in, system=s.c_system())
    ref.run(0)
    done = 0
    L = s.hi - s.lo
    for st in (2, 6, 10):
        ref.run(st - done)
        done = st
        g = ref.state()
        xu = g["x"] + g["image"] * L
        x = np.column_stack([fr[st][c] for c in "xyz"])
        assert np.abs(x - xu).max() < 1e-4, st
        f = np.column_stack([fr[st]["f" + c] for c in "xyz"])
        assert np.abs(f - g["f"]).max() < 1e-3 * np.abs(g["f"]).max(), st
    ref.run(2)
    a, b = e.state(), ref.state()
    dx = a["x"] - b["x"]
    dx -= L * np.round(dx / L)
    assert np.abs(dx).max() < 1e-4


@pytest.mark.skipif(not os.path.exists(CLI), reason="gpudpd_b200 not built")
@pytest.mark.parametrize("walls", ["two_wall", "reflect"])
def test_cli_walls_match_reference_executable(walls):
    """Particle walls (fix move, two_wall / wall_reflect), compute wall_contact and a group
    dump compute of the liquid, against the reference executable."""
    from gpumdpd_b200 import inputs
    s = inputs.wall_channel(seed=81, nsteps=10, thermo=1, walls=walls)
    run_in = re.sub(r"(?m)^read_data .*$", "read_data system.data", s.run_in)
    run_in += "compute cd liquid dump 5 liquid.trj\n"
    files = ["thermo.txt", "wall_contact.txt", "liquid.trj"]
    ours = _run(CLI, s, run_in, files)
    assert set(ours) == set(files)
    fr = parse_trj_text(ours["liquid.trj"])
    assert sorted(fr) == [0, 5, 10]
    liquid = np.flatnonzero(s.types == 1) + 1
    for st, f in fr.items():
        assert f["cols"] == ["id", "type", "x", "y", "z"]
        np.testing.assert_array_equal(f["id"], liquid)
    h, wc = _thermo(ours["wall_contact.txt"])
    assert h == ["step", "wall_contact"] and list(wc["step"]) == list(range(11))
    if not os.path.exists(STOCK):
        pytest.skip("reference build (oracle/build_ref.sh SINGLE) not present")
    ref = _run(STOCK, s, run_in, files)
    rh, rwc = _thermo(ref["wall_contact.txt"])
    assert rh == h
    assert wc["wall_contact"][0] == rwc["wall_contact"][0]
    assert np.abs(wc["wall_contact"] - rwc["wall_contact"]).max() <= 1
    rfr = parse_trj_text(ref["liquid.trj"])
    assert sorted(rfr) == sorted(fr)
    for st in fr:
        np.testing.assert_array_equal(rfr[st]["id"], fr[st]["id"])
        d = np.column_stack([fr[st][c] - rfr[st][c] for c in "xyz"])
        d -= (s.hi - s.lo) * np.round(d / (s.hi - s.lo))
        assert np.abs(d).max() < (2e-6 if st == 0 else 5e-5), st
    _, th = _thermo(ours["thermo.txt"])
    _, rth = _thermo(ref["thermo.txt"])
    assert th["temp"][0] == pytest.approx(rth["temp"][0], rel=2e-5)
    np.testing.assert_allclose(th["temp"], rth["temp"], rtol=2e-3)


@pytest.mark.skipif(not os.path.exists(CLI), reason="gpudpd_b200 not built")
def test_cli_molecular_compute_dump():
    """A dump compute of a bonded system lists id mol type x y z (compute_dump.cu:110-128)."""
    from gpumdpd_b200 import inputs
    s = inputs.diblock_melt(L=6.0, seed=83, nsteps=4, thermo=2)
    run_in = re.sub(r"(?m)^read_data .*$", "read_data system.data", s.run_in)
    run_in = run_in.replace("group all type 1 2", "group all type 1 2\ngroup heads type 1")
    run_in += "compute cd heads dump 2 heads.trj\n"
    ours = _run(CLI, s, run_in, ["heads.trj"])
    fr = parse_trj_text(ours["heads.trj"])
    assert sorted(fr) == [0, 2, 4]
    assert fr[0]["cols"] == ["id", "mol", "type", "x", "y", "z"]
    np.testing.assert_array_equal(fr[0]["id"], np.flatnonzero(s.types == 1) + 1)
    np.testing.assert_array_equal(fr[0]["mol"], s.mol[s.types == 1])
    if os.path.exists(STOCK):
        ref = _run(STOCK, s, run_in, ["heads.trj"])
        rfr = parse_trj_text(ref["heads.trj"])
        assert sorted(rfr) == sorted(fr)
        np.testing.assert_array_equal(rfr[0]["mol"], fr[0]["mol"])
        np.testing.assert_allclose(np.column_stack([fr[0][c] for c in "xyz"]),
                                   np.column_stack([rfr[0][c] for c in "xyz"]), atol=2e-6)


DOUBLE = os.path.join(ROOT, "oracle", "_ref", "gpudpd_double")


def _block_mean(x, nb=10):
    b = np.array([c.mean() for c in np.array_split(np.asarray(x), nb)])
    return b.mean(), b.std(ddof=1) / np.sqrt(nb)


@pytest.mark.skipif(not (os.path.exists(CLI) and os.path.exists(DOUBLE)),
                    reason="gpudpd_b200 or the reference's -DDOUBLE build not present")
@pytest.mark.parametrize("name", ["dpd", "diblock"])
def test_fp32_engine_vs_reference_double_build(name):
    """The FP32 engine against the reference's -DDOUBLE build on the same input: the run
    means of T and P agree within their statistical errors (block averages of 10 blocks,
    4 combined standard errors), separating precision from algorithm: the trajectories
    part within tens of steps, the ensembles do not."""
    from gpumdpd_b200 import inputs
    if name == "dpd":
        s = inputs.plain_dpd(L=10.0, seed=91, nsteps=4000, thermo=10)
    else:
        s = inputs.diblock_melt(L=10.0, seed=92, nsteps=4000, thermo=10)
    run_in = re.sub(r"(?m)^read_data .*$", "read_data system.data", s.run_in)
    ours = _thermo(_run(CLI, s, run_in, ["thermo.txt"])["thermo.txt"])[1]
    ref = _thermo(_run(DOUBLE, s, run_in, ["thermo.txt"])["thermo.txt"])[1]
    assert ours["temp"][0] == pytest.approx(ref["temp"][0], rel=1e-5)
    for k in ("temp", "pressure"):
        a, ea = _block_mean(ours[k][100:])
        b, eb = _block_mean(ref[k][100:])
        assert abs(a - b) < 4 * np.hypot(ea, eb) + 1e-3 * abs(b), (k, a, ea, b, eb)


@pytest.mark.skipif(not os.path.exists(DOUBLE), reason="the reference's -DDOUBLE build not present")
@pytest.mark.parametrize("name", ["dpd", "diblock"])
def test_fp64_engine_vs_reference_double_build(name):
    """The FP64 parity engine against the reference's -DDOUBLE build on the same input: the
    thermo rows of the first 20 steps agree to thermo.txt's print precision (6 decimals; the
    diblock's bond PE, about 1e4, to 2e-10 relative), where the FP32 engine parts from it
    within a few steps; later the two FP64 trajectories part too (2e-8 relative in the bond
    PE by step 35), and the 4000-step run means of T and P agree within their statistical
    errors."""
    from gpumdpd_b200 import Engine, inputs
    if name == "dpd":
        s = inputs.plain_dpd(L=10.0, seed=91, nsteps=4000, thermo=1)
    else:
        s = inputs.diblock_melt(L=10.0, seed=92, nsteps=4000, thermo=1)
    run_in = re.sub(r"(?m)^read_data .*$", "read_data system.data", s.run_in)
    ref = _thermo(_run(DOUBLE, s, run_in, ["thermo.txt"])["thermo.txt"])[1]
    e = Engine(s.run_in, system=s.c_system(), precision="fp64")
    e.run(4000)
    ours = e.thermo(max_rows=5000)
    assert len(ours["step"]) == len(ref["temp"]) == 4001
    cols = ["temp", "pressure"] + (["bond_pe"] if name == "diblock" else [])
    for k in cols:
        np.testing.assert_allclose(ours[k][:21], ref[k][:21], rtol=0, atol=2e-6)
    for k in ("temp", "pressure"):
        a, ea = _block_mean(ours[k][100:])
        b, eb = _block_mean(ref[k][100:])
        assert abs(a - b) < 4 * np.hypot(ea, eb) + 1e-3 * abs(b), (k, a, ea, b, eb)


@pytest.mark.skipif(not (os.path.exists(CLI) and os.path.exists(DOUBLE)),
                    reason="gpudpd_b200 or the reference's -DDOUBLE build not present")
def test_cli_fp64_vs_reference_double_executable():
    """`gpudpd_b200 --fp64` in place of the reference's -DDOUBLE executable: the same
    thermo.txt columns, rows agreeing to print precision over the first 20 steps, and a
    write_data file with the same atoms."""
    from gpumdpd_b200 import inputs
    s = inputs.diblock_melt(L=8.0, seed=93, nsteps=60, thermo=1)
    run_in = re.sub(r"(?m)^read_data .*$", "read_data system.data", s.run_in) + "write_data out.data\n"
    ours = _run(CLI, s, run_in, ["thermo.txt", "out.data"], args=["--fp64"])
    ref = _run(DOUBLE, s, run_in, ["thermo.txt", "out.data"])
    ho, to = _thermo(ours["thermo.txt"])
    hr, tr = _thermo(ref["thermo.txt"])
    assert ho == hr
    assert len(to["step"]) == len(tr["step"]) == 61
    for k in hr:
        np.testing.assert_allclose(to[k][:21], tr[k][:21], rtol=0, atol=2e-6, err_msg=k)
    assert "out.data" in ours and len(ours["out.data"].splitlines()) == len(ref["out.data"].splitlines())
