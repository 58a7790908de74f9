"""ctypes binding of the FP64 CPU oracle (oracle/dpd_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference legs as the checker; the product never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "liboracle.so")
MAXT = 32


class OracleFF(ctypes.Structure):
    _fields_ = [
        ("style", ctypes.c_int), ("ntypes", ctypes.c_int), ("kT", ctypes.c_double),
        ("dt", ctypes.c_double), ("seed", ctypes.c_uint32),
        ("coeff", (ctypes.c_double * 5) * (MAXT * MAXT)), ("mass", ctypes.c_double * MAXT),
        ("bond_style", ctypes.c_int), ("nbondtypes", ctypes.c_int),
        ("bond_coeff", (ctypes.c_double * 4) * MAXT),
        ("angle_style", ctypes.c_int), ("nangletypes", ctypes.c_int),
        ("angle_coeff", (ctypes.c_double * 2) * MAXT),
        ("spring_on", ctypes.c_int), ("spring_mask", ctypes.c_uint32), ("spring_k", ctypes.c_double),
        ("spring_c", ctypes.c_double * 3), ("spring_r0", ctypes.c_double),
        ("rvcm_on", ctypes.c_int), ("rvcm_mask", ctypes.c_uint32), ("rvcm_freq", ctypes.c_uint32),
        ("rvcm_flag", ctypes.c_int * 3),
        ("recenter_on", ctypes.c_int), ("recenter_mask", ctypes.c_uint32), ("recenter_freq", ctypes.c_uint32),
        ("recenter_c", ctypes.c_double * 3),
        ("integ_mask", ctypes.c_uint32),
        ("n_move", ctypes.c_int), ("move_mask", ctypes.c_uint32 * 4), ("move_v", (ctypes.c_double * 3) * 4),
        ("n_reflect", ctypes.c_int), ("refl_mask", ctypes.c_uint32 * 4), ("refl_dir", ctypes.c_int * 4),
        ("refl_lo", ctypes.c_double * 4), ("refl_hi", ctypes.c_double * 4),
        ("n_twowall", ctypes.c_int), ("tw_mask", ctypes.c_uint32 * 2), ("tw_lo", ctypes.c_uint32 * 2),
        ("tw_hi", ctypes.c_uint32 * 2), ("tw_dir", ctypes.c_int * 2),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    lib = ctypes.CDLL(LIB)
    vp, i, u32, d, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_double, ctypes.c_long
    lib.oracle_saru.restype = ctypes.c_float
    lib.oracle_saru.argtypes = [u32, u32, u32, ctypes.c_int32]
    lib.oracle_set_saru_double_tail.restype = None
    lib.oracle_set_saru_double_tail.argtypes = [i]
    lib.oracle_spring_last.restype = None
    lib.oracle_spring_last.argtypes = [vp]
    lib.oracle_set_angles.restype = None
    lib.oracle_set_angles.argtypes = [i, vp]
    lib.oracle_saru_batch.restype = None
    lib.oracle_saru_batch.argtypes = [i, vp, vp, u32, vp, vp]
    lib.oracle_pairs_f64.restype = i64
    lib.oracle_pairs_f64.argtypes = [i, vp, vp, vp, vp, d, vp, i64]
    lib.oracle_pairs_f32.restype = i64
    lib.oracle_pairs_f32.argtypes = [i, vp, vp, vp, vp, vp, ctypes.c_float, vp, i64]
    lib.oracle_forces.restype = i
    lib.oracle_forces.argtypes = [i, vp, vp, vp, vp, vp, vp, ctypes.POINTER(OracleFF), u32, i, vp, vp,
                                  vp, vp, vp]
    lib.oracle_run.restype = i
    lib.oracle_run.argtypes = [i, vp, vp, vp, vp, vp, vp, vp, ctypes.POINTER(OracleFF), i, vp, u32, i,
                               i, u32, vp, vp, i, vp, vp]
    lib.oracle_rdf.restype = i
    lib.oracle_rdf.argtypes = [i, vp, vp, vp, vp, i, i, d, i, vp]
    lib.oracle_bench_steps.restype = i
    lib.oracle_bench_steps.argtypes = [i, vp, vp, vp, vp, vp, vp, ctypes.POINTER(OracleFF), i, vp,
                                       u32, i, d, i]
    assert lib.oracle_ff_size() == ctypes.sizeof(OracleFF)
    _lib = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def tri_index(ti, tj, nt):
    a, b = min(ti, tj), max(ti, tj)
    return ((a - 1) * nt - (a - 1) * (a - 2) // 2 + b - a + 1) - 1


def make_ff(style, ntypes, coeffs, kT, dt, seed, masses, bond_style=0, bond_coeffs=(), angle_style=0,
            angle_coeffs=()):
    """coeffs: {(ti,tj): (A, B, gamma, rc, rd)}; bond_coeffs: list of 4-tuples."""
    ff = OracleFF()
    ff.style = style
    ff.ntypes = ntypes
    ff.kT = kT
    ff.dt = dt
    ff.seed = seed
    for (ti, tj), c in coeffs.items():
        idx = tri_index(ti, tj, ntypes)
        for k in range(5):
            ff.coeff[idx][k] = c[k]
    for t, m in enumerate(masses):
        ff.mass[t] = m
    ff.bond_style = bond_style
    ff.nbondtypes = len(bond_coeffs)
    for b, c in enumerate(bond_coeffs):
        for k in range(len(c)):
            ff.bond_coeff[b][k] = c[k]
    ff.angle_style = angle_style
    ff.nangletypes = len(angle_coeffs)
    for a, c in enumerate(angle_coeffs):
        ff.angle_coeff[a][0], ff.angle_coeff[a][1] = c[0], c[1]
    return ff


def ff_from_run_in(text, masses):
    """Force field of a run.in text (pair_style/pair_coeff/bond_style/bond_coeff/timestep)."""
    style, kT, rc, rd, seed, dt = 0, 1.0, 1.0, 0.0, 0, 0.01
    coeffs, bonds, bstyle, angles, astyle = {}, {}, 0, {}, 0
    raw = []
    for line in text.splitlines():
        t = line.split("#")[0].split()
        if t:
            raw.append(t)
    for t in raw:
        if t[0] == "timestep":
            dt = float(t[1])
        if t[0] == "pair_style":
            if t[1] == "dpd":
                style, kT, rc, seed = 0, float(t[2]), float(t[3]), int(t[4])
            else:
                style, kT, rc, rd, seed = 1, float(t[2]), float(t[3]), float(t[4]), int(t[5])
        if t[0] == "bond_style":
            bstyle = {"harmonic": 1, "fene": 2}[t[1]]
        if t[0] == "angle_style":
            astyle = {"harmonic": 1}[t[1]]
    for t in raw:
        if t[0] == "pair_coeff":
            ti, tj = int(t[1]), int(t[2])
            if style == 0:
                A, g = float(t[3]), float(t[4])
                r = float(t[5]) if len(t) > 5 else rc
                coeffs[(ti, tj)] = (A, 0.0, g, r, 0.0)
            else:
                A, B, g = float(t[3]), float(t[4]), float(t[5])
                r, d = (float(t[6]), float(t[7])) if len(t) > 6 else (rc, rd)
                coeffs[(ti, tj)] = (A, B, g, r, d)
        if t[0] == "bond_coeff":
            bonds[int(t[1])] = tuple(float(v) for v in t[2:])
        if t[0] == "angle_coeff":
            angles[int(t[1])] = (float(t[2]), float(t[3]))
    bc = [bonds[k] for k in sorted(bonds)]
    ac = [angles[k] for k in sorted(angles)]
    ff = make_ff(style, len(masses), coeffs, kT, dt, seed, masses, bstyle, bc, astyle, ac)
    # groups and the group fixes (spring, rvcm, recenter)
    groups = {t[1]: [int(v) for v in t[3:]] for t in raw if t[0] == "group" and len(t) > 3}
    def mask(g):
        m = 0
        for ty in groups[g]:
            m |= 1 << (ty - 1)
        return m
    for t in raw:
        if t[0] != "fix" or len(t) < 4:
            continue
        if t[3] == "spring":
            ff.spring_on, ff.spring_mask, ff.spring_k = 1, mask(t[2]), float(t[4])
            for d in range(3):
                ff.spring_c[d] = float(t[5 + d])
            ff.spring_r0 = float(t[8])
        elif t[3] == "rvcm":
            ff.rvcm_on, ff.rvcm_mask, ff.rvcm_freq = 1, mask(t[2]), int(t[4])
            for d in range(3):
                ff.rvcm_flag[d] = int(t[5 + d])
        elif t[3] == "recenter":
            ff.recenter_on, ff.recenter_mask, ff.recenter_freq = 1, mask(t[2]), int(t[4])
            for d in range(3):
                ff.recenter_c[d] = float(t[5 + d])
        elif t[3] == "nve":
            ff.integ_mask |= mask(t[2])
        elif t[3] == "move":
            k = ff.n_move
            ff.move_mask[k] = mask(t[2])
            for d in range(3):
                ff.move_v[k][d] = float(t[4 + d])
            ff.n_move = k + 1
        elif t[3] == "wall_reflect":
            k = ff.n_reflect
            ff.refl_mask[k], ff.refl_lo[k], ff.refl_hi[k] = mask(t[2]), float(t[4]), float(t[5])
            ff.refl_dir[k] = "xyz".index(t[6])
            ff.n_reflect = k + 1
        elif t[3] == "two_wall":
            k = ff.n_twowall
            ff.tw_mask[k], ff.tw_lo[k], ff.tw_hi[k] = mask(t[2]), mask(t[4]), mask(t[5])
            ff.tw_dir[k] = "xyz".index(t[6])
            ff.n_twowall = k + 1
    return ff


def set_saru_double_tail(on):
    """Evaluate Saru's tail as the reference's -DDOUBLE build does (golden tests only)."""
    load().oracle_set_saru_double_tail(1 if on else 0)


def saru(t1, t2, seed, step):
    lib = load()
    t1 = np.ascontiguousarray(t1, dtype=np.uint32)
    t2 = np.ascontiguousarray(t2, dtype=np.uint32)
    st = np.ascontiguousarray(np.broadcast_to(step, t1.shape), dtype=np.int32)
    out = np.empty(t1.shape, dtype=np.float32)
    lib.oracle_saru_batch(len(t1), _p(t1), _p(t2), seed, _p(st), _p(out))
    return out


def _set_angles(lib, angles):
    a = None if angles is None else np.ascontiguousarray(angles, dtype=np.int32)
    lib.oracle_set_angles(0 if a is None else len(a), _p(a))
    return a


def forces(ff, tags, types, x, v, lo, L, step, bonds=None, angles=None):
    lib = load()
    keep = _set_angles(lib, angles)
    n = len(types)
    tags = np.ascontiguousarray(tags, dtype=np.int32)
    types = np.ascontiguousarray(types, dtype=np.int32)
    x = np.ascontiguousarray(x, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    lo = np.ascontiguousarray(lo, dtype=np.float64)
    L = np.ascontiguousarray(L, dtype=np.float64)
    f = np.empty((n, 3))
    rho = np.empty(n)
    en = np.empty(3)
    vir = np.empty(6)
    nb = 0 if bonds is None else len(bonds)
    b = None if bonds is None else np.ascontiguousarray(bonds, dtype=np.int32)
    st = lib.oracle_forces(n, _p(tags), _p(types), _p(x), _p(v), _p(lo), _p(L), ctypes.byref(ff), step,
                           nb, _p(b), _p(f), _p(rho), _p(en), _p(vir))
    lib.oracle_set_angles(0, None)
    del keep
    return {"f": f, "rho": rho, "pair_pe": en[0], "bond_pe": en[1], "angle_pe": en[2], "virial": vir,
            "status": st}


def run(ff, tags, types, x, v, lo, L, first_step, nsteps, log_f, bonds=None, zero_step=True, f0=None,
        angles=None):
    """Velocity-Verlet in FP64; returns final state and logged thermo rows.  Without a zero
    step, f0 are the forces of step first_step-1 (used by the first half kick)."""
    lib = load()
    keep = _set_angles(lib, angles)
    n = len(types)
    tags = np.ascontiguousarray(tags, dtype=np.int32)
    types = np.ascontiguousarray(types, dtype=np.int32)
    x = np.array(x, dtype=np.float64, order="C")
    v = np.array(v, dtype=np.float64, order="C")
    img = np.zeros((n, 3), dtype=np.int32)
    lo = np.ascontiguousarray(lo, dtype=np.float64)
    L = np.ascontiguousarray(L, dtype=np.float64)
    maxlog = nsteps + 2
    th = np.zeros((maxlog, 12))
    ls = np.zeros(maxlog, dtype=np.int32)
    f = np.zeros((n, 3)) if f0 is None else np.array(f0, dtype=np.float64, order="C")
    rho = np.zeros(n)
    nb = 0 if bonds is None else len(bonds)
    b = None if bonds is None else np.ascontiguousarray(bonds, dtype=np.int32)
    nlog = lib.oracle_run(n, _p(tags), _p(types), _p(x), _p(v), _p(img), _p(lo), _p(L), ctypes.byref(ff),
                          nb, _p(b), first_step, nsteps, 1 if zero_step else 0, log_f, _p(th), _p(ls),
                          maxlog, _p(f), _p(rho))
    lib.oracle_set_angles(0, None)
    del keep
    if nlog < 0:
        raise RuntimeError(f"oracle_run failed: {nlog}")
    cols = ["temp", "pair_pe", "bond_pe", "pressure", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz", "ke",
            "angle_pe"]
    thermo = {c: th[:nlog, k] for k, c in enumerate(cols)}
    thermo["step"] = ls[:nlog]
    return {"x": x, "v": v, "image": img, "f": f, "rho": rho, "thermo": thermo}


def spring_last():
    """{Fx, Fy, Fz, +-|F|, energy} of the last spring evaluation of `run`/`forces`."""
    lib = load()
    out = np.zeros(5)
    lib.oracle_spring_last(_p(out))
    return out


def pairs_f64(tags, x, lo, L, cut):
    lib = load()
    n = len(tags)
    tags = np.ascontiguousarray(tags, dtype=np.int32)
    x = np.ascontiguousarray(x, dtype=np.float64)
    lo = np.ascontiguousarray(lo, dtype=np.float64)
    L = np.ascontiguousarray(L, dtype=np.float64)
    cnt = lib.oracle_pairs_f64(n, _p(tags), _p(x), _p(lo), _p(L), cut, None, 0)
    out = np.empty((max(cnt, 1), 2), dtype=np.int32)
    lib.oracle_pairs_f64(n, _p(tags), _p(x), _p(lo), _p(L), cut, _p(out), cnt)
    return out[:cnt]


def pairs_f32(tags, cell, off, nc, w, cut2):
    lib = load()
    n = len(tags)
    tags = np.ascontiguousarray(tags, dtype=np.int32)
    cell = np.ascontiguousarray(cell, dtype=np.int32)
    off = np.ascontiguousarray(off, dtype=np.float32)
    nc = np.ascontiguousarray(nc, dtype=np.int32)
    w = np.ascontiguousarray(w, dtype=np.float32)
    cnt = lib.oracle_pairs_f32(n, _p(tags), _p(cell), _p(off), _p(nc), _p(w), float(cut2), None, 0)
    out = np.empty((max(cnt, 1), 2), dtype=np.int32)
    lib.oracle_pairs_f32(n, _p(tags), _p(cell), _p(off), _p(nc), _p(w), float(cut2), _p(out), cnt)
    return out[:cnt]


def rdf(types, x, lo, L, ta, tb, rmax, nbins):
    lib = load()
    types = np.ascontiguousarray(types, dtype=np.int32)
    x = np.ascontiguousarray(x, dtype=np.float64)
    g = np.empty(nbins)
    lib.oracle_rdf(len(types), _p(types), _p(x), _p(np.asarray(lo, dtype=np.float64)),
                   _p(np.asarray(L, dtype=np.float64)), ta, tb, rmax, nbins, _p(g))
    return g


def bench_steps(ff, tags, types, x, v, lo, L, first_step, nsteps, skin, nthreads, bonds=None):
    """The reference algorithm (half Verlet list + skin) in FP64 on nthreads host threads;
    bonds (rows type, tag_i, tag_j) add their forces on one thread."""
    lib = load()
    tags = np.ascontiguousarray(tags, dtype=np.int32)
    types = np.ascontiguousarray(types, dtype=np.int32)
    x = np.array(x, dtype=np.float64, order="C")
    v = np.array(v, dtype=np.float64, order="C")
    nb, bp = 0, None
    if bonds is not None and len(bonds):
        bonds = np.ascontiguousarray(bonds, dtype=np.int32)
        nb, bp = len(bonds), _p(bonds)
    return lib.oracle_bench_steps(len(types), _p(tags), _p(types), _p(x), _p(v),
                                  _p(np.asarray(lo, dtype=np.float64)), _p(np.asarray(L, dtype=np.float64)),
                                  ctypes.byref(ff), nb, bp, first_step, nsteps, skin, nthreads)
