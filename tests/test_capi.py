"""The C-ABI boundary on a host without a GPU: the library loads, exports every symbol
declared in include/dpd_b200.h, applies the reference's run.in grammar and data-file
checks (src/main/read_in.cu:40-371, plugin isEnabled/validateParams) before touching
a device, and refuses to run without one (no CPU fallback)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def _header_symbols():
    text = open(os.path.join(ROOT, "include", "dpd_b200.h")).read()
    return sorted(set(re.findall(r"\b(dpd_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from gpumdpd_b200 import capi
    lib = capi.load()
    syms = _header_symbols()
    assert len(syms) >= 30
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(capi.EXPORTED)


def _create(run_in, system):
    from gpumdpd_b200 import capi
    lib = capi.load()
    h = ctypes.c_void_p()
    s, keep = system.c_system()
    code = lib.dpd_create_from_system(run_in.encode(), ctypes.byref(s), ctypes.byref(h))
    msg = lib.dpd_last_error(None).decode()
    if code == 0:
        lib.dpd_destroy(h)
    return code, msg


@pytest.fixture(scope="module")
def base():
    from gpumdpd_b200 import inputs
    return inputs.plain_dpd(L=6.0, seed=1)


def _no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(not _no_gpu(), reason="checks the no-device refusal")
def test_valid_input_refuses_without_gpu(base):
    code, msg = _create(base.run_in, base)
    assert code == -8 and "no CPU fallback" in msg


def _create_fp64(run_in, system):
    from gpumdpd_b200 import capi
    lib = capi.load()
    h = ctypes.c_void_p()
    s, keep = system.c_system()
    code = lib.dpd_create_fp64(run_in.encode(), None, None, ctypes.byref(s), ctypes.byref(h))
    msg = lib.dpd_last_error(None).decode()
    if code == 0:
        lib.dpd_destroy(h)
    return code, msg


def test_fp64_mode_checks():
    """The FP64 parity engine applies the same grammar checks, refuses the fixes, computes
    and dumps it does not cover before touching a device, and has no CPU fallback."""
    from gpumdpd_b200 import inputs
    s = inputs.probe_fixes(L=9.0, seed=5, nsteps=10, thermo=1)
    code, msg = _create_fp64(s.run_in, s)
    assert code == -1 and "FP64 parity mode" in msg
    b = inputs.plain_dpd(L=6.0, seed=1)
    code, msg = _create_fp64(b.run_in.replace("run 1000\n", ""), b)
    assert code == -1 and "run command is missing" in msg
    code, msg = _create_fp64(b.run_in + "compute ct all temp 1 t.txt\n", b)
    assert code == -1 and "FP64 parity mode" in msg
    if _no_gpu():
        code, msg = _create_fp64(b.run_in, b)
        assert code == -8 and "no CPU fallback" in msg


BAD = [
    ("unknown", lambda t: t + "foo 1 2\n", "unknown command foo"),
    ("no_run", lambda t: t.replace("run 1000\n", ""), "run command is missing"),
    ("no_thermo", lambda t: t.replace("thermo 100\n", ""), "thermo command is missing"),
    ("no_atom_style", lambda t: t.replace("atom_style atomic\n", ""), "atom_style command is missing"),
    ("neighbor_args", lambda t: t.replace("neighbor 1.0 0.3 10.0 1", "neighbor 1.0 0.3 10.0"), "illegal neighbor command"),
    ("nl_f_float", lambda t: t.replace("neighbor 1.0 0.3 10.0 1", "neighbor 1.0 0.3 10.0 1.5"), "illegal neighbor command"),
    ("pair_args", lambda t: t.replace("pair_style dpd 1.0 1.0 1", "pair_style dpd 1.0 1.0"), "illegal pair_style dpd"),
    ("rc_too_big", lambda t: t.replace("pair_style dpd 1.0 1.0 1", "pair_style dpd 1.0 1.5 1"), "global rc should not be bigger"),
    ("coeff_missing", lambda t: t.replace("pair_coeff 1 1 25.0 4.5\n", ""), "all pair_coeff are not set"),
    ("coeff_order", lambda t: t.replace("pair_coeff 1 1 25.0 4.5", "pair_coeff 2 1 25.0 4.5"), "typei <= typej"),
    ("no_pair_style", lambda t: t.replace("pair_style dpd 1.0 1.0 1\n", ""), "pair_style command is missing"),
    ("two_pair_styles", lambda t: t + "pair_style mdpd 1.0 1.0 0.75 3\n", "more than one enabled pair_style"),
    ("group_type", lambda t: t.replace("group all type 1", "group all type 2"), "Type in group is not included"),
    ("group_dup", lambda t: t + "group all type 1\n", "already exists"),
    ("fix_group", lambda t: t.replace("fix md all nve", "fix md none nve"), "Group 'none' not found"),
    ("fix_style", lambda t: t.replace("fix md all nve", "fix md all langevin"), "Fix type 'langevin' not found"),
    ("fix_params", lambda t: t.replace("fix md all nve", "fix md all nve 1"), "illegal fix_nve command"),
    ("fix_dup_id", lambda t: t + "fix md all nve\n", "already registered"),
    ("dump_args", lambda t: t + "dump 0 10 wrapped force_no\n", "illegal dump command"),
    ("compute_bad", lambda t: t + "compute c all foo 1 x.txt\n", "Compute type 'foo' not found"),
    ("angle", lambda t: t.replace("atom_style atomic", "atom_style angle") + "bond_style harmonic\n", "angle_style command is missing"),
]


@pytest.mark.parametrize("name,edit,msg", BAD, ids=[b[0] for b in BAD])
def test_run_in_grammar_errors(base, name, edit, msg):
    text = base.run_in.replace("pair_style dpd 1.0 1.0 2", "pair_style dpd 1.0 1.0 1")
    text = re.sub(r"pair_style dpd 1\.0 1\.0 \d+", "pair_style dpd 1.0 1.0 1", text)
    code, err = _create(edit(text), base)
    assert code == -1, err
    assert msg in err


def test_mdpd_rd_checks(base):
    from gpumdpd_b200 import inputs
    s = inputs.mdpd_slab(Lx=6, Ly=6, Lz=12, z0=3, z1=9)
    code, err = _create(s.run_in.replace("mdpd 1.0 1.0 0.75", "mdpd 1.0 1.0 1.25"), s)
    assert code == -1 and "rd should not be bigger than rc" in err
    code, err = _create(s.run_in.replace("pair_coeff 1 1 -40.0 25.0 4.5", "pair_coeff 1 1 -40.0 25.0"), s)
    assert code == -1 and "illegal pair_coeff command for pair mdpd" in err


def test_bond_style_checks():
    from gpumdpd_b200 import inputs
    s = inputs.diblock_melt(L=6.0, seed=1)
    code, err = _create(s.run_in.replace("bond_coeff 1 4.0 0.0\n", ""), s)
    assert code == -1 and "all bond_coeff are not set" in err
    code, err = _create(s.run_in.replace("bond_style harmonic\n", ""), s)
    assert code == -1 and "bond_style command is missing" in err
    code, err = _create(s.run_in.replace("bond_coeff 1 4.0 0.0", "bond_coeff 1 4.0"), s)
    assert code == -1 and "bond_style harmonic" in err


def test_angle_style_checks():
    """atom_style angle needs angle_style harmonic and every angle_coeff (reference messages,
    src/main/read_in.cu:347-371, src/force/angle_harmonic.cu:19-147)."""
    from gpumdpd_b200 import inputs
    s = inputs.angle_chains(L=6.0, seed=2)
    code, err = _create(s.run_in.replace("angle_style harmonic\n", ""), s)
    assert code == -1 and "angle_style command is missing" in err
    code, err = _create(s.run_in.replace("angle_coeff 1 2.0 180.0", "angle_coeff 1 2.0"), s)
    assert code == -1 and "angle_coeff" in err
    code, err = _create(s.run_in.replace("angle_coeff 1 2.0 180.0\n", ""), s)
    assert code == -1 and "all angle_coeff are not set" in err
    code, err = _create(s.run_in.replace("angle_style harmonic", "angle_style cosine"), s)
    assert code == -1 and "angle_style" in err
    code, err = _create(s.run_in, s)
    assert code in (0, -8), err


def test_data_file_reader(tmp_path, base):
    """Files in the reference's write_data layout are read (and bad ones rejected)."""
    from gpumdpd_b200 import capi, inputs
    lib = capi.load()
    for s in (base, inputs.diblock_melt(L=6.0, seed=2), inputs.angle_chains(L=6.0, seed=3)):
        p = tmp_path / "in.data"
        s.write_data(str(p))
        h = ctypes.c_void_p()
        code = lib.dpd_create(s.run_in.encode(), str(p).encode(), None, ctypes.byref(h))
        err = lib.dpd_last_error(None).decode()
        assert code in (0, -8), err
        if code == 0:
            lib.dpd_destroy(h)
    # duplicate atom id
    p = tmp_path / "bad.data"
    base.write_data(str(p))
    lines = open(p).read().splitlines()
    k = next(i for i, l in enumerate(lines) if l.startswith("Atoms")) + 3
    lines[k] = "1 " + " ".join(lines[k].split()[1:])
    open(p, "w").write("\n".join(lines) + "\n")
    h = ctypes.c_void_p()
    code = lib.dpd_create(base.run_in.encode(), str(p).encode(), None, ctypes.byref(h))
    assert code == -1 and "Atoms section" in lib.dpd_last_error(None).decode()
    code = lib.dpd_create(base.run_in.encode(), b"/nonexistent/file.data", None, ctypes.byref(h))
    assert code == -2


def test_inputs_generators():
    from gpumdpd_b200 import inputs
    s = inputs.plain_dpd()
    assert s.n == 3000 and np.all((s.x >= 0) & (s.x < 10))
    assert np.abs((s.v).sum(axis=0)).max() < 1e-9
    m = inputs.diblock_melt(L=10.0)
    assert m.n == 3000 and len(m.bonds) == 2700
    assert list(m.types[:10]) == [1] * 5 + [2] * 5
    b = np.linalg.norm(((m.x[m.bonds[:, 1] - 1] - m.x[m.bonds[:, 2] - 1]) + 5) % 10 - 5, axis=1)
    assert np.allclose(b, 0.9)
    sl = inputs.mdpd_slab()
    assert sl.n == 384000 and sl.x[:, 2].min() >= 40 and sl.x[:, 2].max() <= 80
    reps = inputs.replica_sweep(n_rep=8, nsteps=10)
    ns = [r.n for r in reps]
    assert min(ns) >= 3 * 8 ** 3 * 0.99 and max(ns) <= 3 * 24 ** 3 * 1.01


def test_group_fix_checks():
    """fix spring / rvcm / recenter parameters (validateParams of src/fix/fix_spring.cu:17-52,
    fix_rvcm.cu:17-40, fix_recenter.cu:17-32) and the in-box checks of their preprocess."""
    from gpumdpd_b200 import inputs
    s = inputs.probe_fixes(L=6.0, seed=2, radius=1.0)
    code, err = _create(s.run_in, s)
    assert code in (0, -8), err
    t = s.run_in
    spring = [ln for ln in t.splitlines() if " spring " in ln][0]
    rvcm = [ln for ln in t.splitlines() if " rvcm " in ln][0]
    rec = [ln for ln in t.splitlines() if " recenter " in ln][0]
    cases = [
        (t.replace(spring, spring.rsplit(" ", 3)[0]), "illegal fix_spring command"),
        (t.replace(spring, spring.replace("spring 50.0 4.0", "spring 50.0 9.5")), "out of the box in x"),
        (t.replace(spring, spring.replace(" spring.txt 2", " spring.txt 0")), "illegal fix_spring command"),
        (t.replace(rvcm, rvcm + " 1"), "illegal fix_rvcm command"),
        (t.replace(rvcm, rvcm.replace("rvcm 3 1 0 1", "rvcm 3 2 0 1")), "illegal fix_rvcm command"),
        (t.replace(rvcm, rvcm.replace("rvcm 3", "rvcm 0")), "illegal fix_rvcm command"),
        (t.replace(rec, rec.replace("recenter 4 3.0 3.0 3.0", "recenter 4 3.0 3.0 7.0")), "out of the box in z"),
        (t.replace(rec, rec.replace("recenter 4", "recenter x")), "illegal fix_recenter command"),
        (t.replace(rec, rec.replace(" probe ", " nogroup ")), "Group 'nogroup' not found"),
        (t + "fix spr2 probe spring 1.0 3.0 3.0 3.0 0.0\n", "at most one fix spring"),
    ]
    for text, msg in cases:
        assert text != t
        code, err = _create(text, s)
        assert code == -1 and msg in err, (msg, err)


def test_group_compute_checks(base):
    """compute temp/rho/msd/tf parameters (validateParams of src/compute/compute_*.cu) and
    the rho region checks (compute_rho.cu:42-75)."""
    t = base.run_in
    ok = t + "compute ct all temp 1 t.txt\ncompute cr all rho 5 0 5 0 5 0 5 r.txt\n" \
             "compute cm all msd 10 m.txt\ncompute cf all tf 2 f.txt\n"
    code, err = _create(ok, base)
    assert code in (0, -8), err
    L = base.hi[0]
    cases = [
        (t + "compute ct all temp 1\n", "illegal compute_temp command"),
        (t + "compute ct all temp 0 t.txt\n", "illegal compute_temp command"),
        (t + "compute cm all msd 1 m.txt x\n", "illegal compute_msd command"),
        (t + "compute cf all tf x f.txt\n", "illegal compute_tf command"),
        (t + "compute cr all rho 1 0 5 0 5 0 r.txt\n", "illegal compute_rho command"),
        (t + "compute cr all rho 1 -1 5 0 5 0 5 r.txt\n", "xlo < box.xlo"),
        (t + f"compute cr all rho 1 0 5 0 5 0 {L + 1} r.txt\n", "zhi > box.zhi"),
        (t + "compute ct all temp 1 t.txt\ncompute ct all msd 1 m.txt\n", "already registered"),
        (t + "".join(f"compute c{k} all temp 1 t{k}.txt\n" for k in range(5)), "at most 4"),
    ]
    for text, msg in cases:
        code, err = _create(text, base)
        assert code == -1 and msg in err, (msg, err)


def test_wall_fix_checks():
    """fix move / wall_reflect / two_wall and compute wall_contact parameters
    (src/fix/fix_move.cu:17-30, fix_wall_reflect.cu:17-80, fix_two_wall.cu:17-40,
    src/compute/compute_wall_contact.cu:17-45)."""
    from gpumdpd_b200 import inputs
    s = inputs.wall_channel(L=6.0, Lz=10.0, seed=3)
    t = s.run_in
    code, err = _create(t, s)
    assert code in (0, -8), err
    r = inputs.wall_channel(L=6.0, Lz=10.0, seed=3, walls="reflect")
    code, err = _create(r.run_in, r)
    assert code in (0, -8), err
    cases = [
        (t.replace("move 0.5 0.0 0.0", "move 0.5 0.0"), "illegal fix_move command"),
        (t.replace("two_wall bottom top z", "two_wall bottom top w"), "Invalid fix_two_wall direction"),
        (t.replace("two_wall bottom top z", "two_wall bottom nowall z"), "Group 'nowall' not found"),
        (t.replace("two_wall bottom top z", "two_wall bottom top"), "illegal fix_two_wall command"),
        (t + "fix wr liquid wall_reflect 5.0 2.0 z\n", "lo_wall_pos should lower than hi_wall_pos"),
        (t + "fix wr liquid wall_reflect -1.0 2.0 z\n", "Wall position is out of the box!"),
        (t + "fix wr liquid wall_reflect 1.0 2.0 q\n", "Invalid fix_wall_reflect direction"),
        (t.replace("wall_contact 1 bottom lo z 1.0", "wall_contact 1 bottom mid z 1.0"), "illegal compute_wall_contact"),
        (t.replace("wall_contact 1 bottom lo z 1.0", "wall_contact 1 nowall lo z 1.0"), "Group 'nowall' not found"),
        (t.replace("wall_contact 1 bottom lo z 1.0 wall_contact.txt", "wall_contact 1 bottom lo z 1.0"),
         "illegal compute_wall_contact"),
    ]
    for text, msg in cases:
        assert text != t
        code, err = _create(text, s)
        assert code == -1 and msg in err, (msg, err)
