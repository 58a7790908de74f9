"""The in-loop drop-in: the reference executable itself (its own integrator, bonds, thermo)
with `pair_style dpd/b200` / `mdpd/b200`, whose Pair plugin hands the reference's device
buffers to dpd_pair_compute_aos, against the same executable with its stock pair style,
on the same input.

Both binaries are built from the reference's unmodified sources by oracle/build_ref.sh
(SINGLE and SHIM).  Stated tolerances: the step-0 thermo row agrees to the printed
precision (1e-5 relative: the same forces up to FP32 summation order), rows up to step 20
within 1e-3, and the means of T and P over the run within 2% (the two FP32 trajectories
separate chaotically after that)."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STOCK = os.path.join(ROOT, "oracle", "_ref", "gpudpd_single")
SHIM = os.path.join(ROOT, "oracle", "_ref", "gpudpd_single_b200")


def _run(binary, system, run_in):
    with tempfile.TemporaryDirectory() as td:
        open(os.path.join(td, "run.in"), "w").write(run_in)
        system.write_data(os.path.join(td, "system.data"))
        p = subprocess.run([binary], cwd=td, capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
        lines = open(os.path.join(td, "thermo.txt")).read().split("\n")
    head = lines[0].split()
    rows = np.array([[float(v) for v in ln.split()] for ln in lines[1:] if ln.strip()])
    return {k: rows[:, i] for i, k in enumerate(head)}


def _case(name):
    from gpumdpd_b200 import inputs
    if name == "dpd":
        s = inputs.plain_dpd(L=10.0, seed=2024, nsteps=100, thermo=5)
        style = "dpd"
    elif name == "diblock":
        s = inputs.diblock_melt(L=10.0, seed=5, nsteps=100, thermo=5)
        style = "dpd"
    elif name == "angles":
        s = inputs.angle_chains(L=8.0, seed=29, nsteps=100, thermo=5, angle_k=3.0, theta0=120.0)
        style = "dpd"
    else:
        s = inputs.mdpd_slab(Lx=8.0, Ly=8.0, Lz=24.0, z0=8.0, z1=16.0, seed=11, nsteps=100, thermo=5)
        style = "mdpd"
    run_in = re.sub(r"(?m)^read_data .*$", "read_data system.data", s.run_in)
    return s, run_in, style


@pytest.mark.skipif(not (os.path.exists(STOCK) and os.path.exists(SHIM)),
                    reason="reference builds (oracle/build_ref.sh SINGLE and SHIM) not present")
@pytest.mark.parametrize("name", ["dpd", "diblock", "angles", "mdpd"])
def test_reference_loop_with_b200_pair_style(name):
    s, run_in, style = _case(name)
    stock = _run(STOCK, s, run_in)
    ours = _run(SHIM, s, run_in.replace(f"pair_style {style} ", f"pair_style {style}/b200 "))
    assert np.array_equal(stock["step"], ours["step"])
    for k in ("temp", "pair_pe", "pressure"):
        a, b = stock[k], ours[k]
        assert abs(a[0] - b[0]) <= 1e-5 * abs(a[0]) + 2e-6, (k, a[0], b[0])
        early = stock["step"] <= 20
        np.testing.assert_allclose(b[early], a[early], rtol=1e-3, atol=1e-5)
    assert ours["temp"].mean() == pytest.approx(stock["temp"].mean(), rel=2e-2)
    assert ours["pressure"].mean() == pytest.approx(stock["pressure"].mean(), rel=2e-2)


def _plugins(run_in, style, which):
    """The run.in with the chosen stock styles replaced by their b200 plugins."""
    if "pair" in which:
        run_in = run_in.replace(f"pair_style {style} ", f"pair_style {style}/b200 ")
    if "bond" in which:
        run_in = run_in.replace("bond_style harmonic", "bond_style harmonic/b200")
    if "nve" in which:
        run_in = re.sub(r"(?m)^(fix \S+ \S+) nve$", r"\1 nve/b200", run_in)
    return run_in


@pytest.mark.skipif(not (os.path.exists(STOCK) and os.path.exists(SHIM)),
                    reason="reference builds (oracle/build_ref.sh SINGLE and SHIM) not present")
@pytest.mark.parametrize("name,which", [("diblock", ("bond",)), ("diblock", ("nve",)),
                                        ("diblock", ("pair", "bond", "nve")), ("angles", ("bond", "nve")),
                                        ("dpd", ("nve",)), ("mdpd", ("pair", "nve"))])
def test_reference_loop_with_b200_bond_and_nve(name, which):
    """bond_style harmonic/b200 (dpd_bond_compute_aos) and fix nve/b200 (dpd_nve_aos) in
    the reference's own loop, alone and together with the pair plugin: the thermo rows
    (bond PE included) follow the stock executable's.  The bond force and the integrator
    repeat the stock FP32 operations, so with the stock pair style the rows agree to the
    printed precision until FP32 atomics reorder sums."""
    s, run_in, style = _case(name)
    stock = _run(STOCK, s, run_in)
    text = _plugins(run_in, style, which)
    assert text != run_in
    ours = _run(SHIM, s, text)
    assert np.array_equal(stock["step"], ours["step"])
    keys = ["temp", "pair_pe", "pressure"] + (["bond_pe"] if "bond_pe" in stock else [])
    for k in keys:
        a, b = stock[k], ours[k]
        assert abs(a[0] - b[0]) <= 1e-5 * abs(a[0]) + 2e-6, (k, a[0], b[0])
        early = stock["step"] <= 20
        np.testing.assert_allclose(b[early], a[early], rtol=1e-3, atol=1e-5)
    assert ours["temp"].mean() == pytest.approx(stock["temp"].mean(), rel=2e-2)
    assert ours["pressure"].mean() == pytest.approx(stock["pressure"].mean(), rel=2e-2)
