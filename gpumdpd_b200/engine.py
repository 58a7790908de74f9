"""Host-side mirror of the reference's simulation surface over the C ABI.

`Engine` corresponds to one GPUDPD run (src/main/main.cu:15-72): it is created from
the text of a run.in (the reference's command grammar) plus a data file or arrays,
advances with :meth:`Engine.run`, and exposes thermo rows (thermo.txt columns),
state, forces, the neighbour list and the RDF.  `Batch` packs many independent
systems into one engine.  Errors raise :class:`DpdError` instead of exiting.
"""
import ctypes

import numpy as np

from . import capi
from .capi import DpdError


def _check(code, lib, handle):
    if code != 0:
        msg = lib.dpd_last_error(handle)
        raise DpdError(code, msg.decode() if msg else "")


def _rows_to_dict(rows, n):
    out = {k: np.empty(n) for k in ("step", "temp", "pair_pe", "bond_pe", "angle_pe", "pressure", "ke")}
    out["p"] = np.empty((n, 6))
    out["momentum"] = np.empty((n, 3))
    for k in range(n):
        r = rows[k]
        out["step"][k] = r.step
        out["temp"][k] = r.temp
        out["pair_pe"][k] = r.pair_pe
        out["bond_pe"][k] = r.bond_pe
        out["angle_pe"][k] = r.angle_pe
        out["pressure"][k] = r.pressure
        out["ke"][k] = r.ke
        out["p"][k] = list(r.p)
        out["momentum"][k] = list(r.momentum)
    out["step"] = out["step"].astype(np.int64)
    return out


class Engine:
    """One DPD system on the GPU (plain engine).

    precision="fp64" makes the FP64 parity engine (the reference's -DDOUBLE build): run,
    thermo, state, set_state and info only; pair, bond and angle styles with fix nve."""

    def __init__(self, run_in, data_path=None, base_dir=None, system=None, precision="fp32"):
        if precision not in ("fp32", "fp64"):
            raise ValueError("precision must be 'fp32' or 'fp64'")
        self.lib = capi.load()
        self.h = ctypes.c_void_p()
        self.precision = precision
        if precision == "fp64":
            s = None
            if system is not None:
                s, self._keep = system
            code = self.lib.dpd_create_fp64(run_in.encode(), data_path.encode() if data_path else None,
                                            base_dir.encode() if base_dir else None,
                                            ctypes.byref(s) if s is not None else None, ctypes.byref(self.h))
        elif system is not None:
            s, self._keep = system
            code = self.lib.dpd_create_from_system(run_in.encode(), ctypes.byref(s), ctypes.byref(self.h))
        else:
            code = self.lib.dpd_create(run_in.encode(), data_path.encode() if data_path else None,
                                       base_dir.encode() if base_dir else None, ctypes.byref(self.h))
        _check(code, self.lib, None)
        n = ctypes.c_int64()
        self.lib.dpd_get_info(self.h, None, None, ctypes.byref(n), None)
        self.n_atoms = n.value

    def close(self):
        if self.h:
            self.lib.dpd_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def run(self, nsteps):
        _check(self.lib.dpd_run(self.h, int(nsteps)), self.lib, self.h)

    def thermo(self, max_rows=4096):
        rows = (capi.dpd_thermo * max_rows)()
        n = ctypes.c_int()
        _check(self.lib.dpd_get_thermo(self.h, rows, max_rows, ctypes.byref(n)), self.lib, self.h)
        return _rows_to_dict(rows, n.value)

    def dump_open(self, path, start=0, every=0, unwrapped=False, force=False, vel=False):
        """Write trajectory frames (the reference's all.trj format) to `path` during later
        runs; every=0 takes the settings of the run.in's dump command."""
        flags = (1 if unwrapped else 0) | (2 if force else 0) | (4 if vel else 0)
        _check(self.lib.dpd_dump_open(self.h, str(path).encode(), int(start), int(every), flags), self.lib, self.h)

    def compute_dump_open(self, compute_id, path=None):
        """Write the frames of the run.in's `compute ID group dump freq file` (to `path`, or
        the compute's file)."""
        _check(self.lib.dpd_compute_dump_open(self.h, str(compute_id).encode(),
                                              str(path).encode() if path else None), self.lib, self.h)

    def dump_close(self):
        _check(self.lib.dpd_dump_close(self.h), self.lib, self.h)

    def compute(self, compute_id, max_rows=2048):
        """Rows of a temp/rho/msd/tf group compute: (n, 2) {step, value} or (n, 4)
        {step, fx, fy, fz}."""
        rows = np.empty((max_rows, 4))
        nc, n = ctypes.c_int(), ctypes.c_int()
        _check(self.lib.dpd_get_compute(self.h, str(compute_id).encode(), capi.ptr(rows), max_rows,
                                        ctypes.byref(nc), ctypes.byref(n)), self.lib, self.h)
        return rows.reshape(-1)[: n.value * nc.value].reshape(n.value, nc.value)

    def write_restart(self, path):
        """Exact checkpoint: FP32 state, forces of the last step, step counter, fix results."""
        _check(self.lib.dpd_write_restart(self.h, str(path).encode()), self.lib, self.h)

    def read_restart(self, path):
        """Resume from a checkpoint of an engine made from the same run.in and system."""
        _check(self.lib.dpd_read_restart(self.h, str(path).encode()), self.lib, self.h)

    def spring_records(self, max_rows=2048):
        """Rows {step, Fx, Fy, Fz, +-|F|, energy} of a `fix spring` with a record file
        (an (n, 6) array; empty without one)."""
        rows = np.empty((max_rows, 6))
        n = ctypes.c_int()
        _check(self.lib.dpd_get_spring_records(self.h, capi.ptr(rows), max_rows, ctypes.byref(n)),
               self.lib, self.h)
        return rows[: n.value]

    def state(self, forces=True, images=True):
        n = self.n_atoms
        x = np.empty((n, 3))
        v = np.empty((n, 3))
        img = np.empty((n, 3), dtype=np.int32) if images else None
        f = np.empty((n, 3)) if forces else None
        _check(self.lib.dpd_get_state(self.h, capi.ptr(x), capi.ptr(v), capi.ptr(img), capi.ptr(f)),
               self.lib, self.h)
        return {"x": x, "v": v, "image": img, "f": f}

    def set_state(self, x, v):
        x = np.ascontiguousarray(x, dtype=np.float64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        _check(self.lib.dpd_set_state(self.h, capi.ptr(x), capi.ptr(v)), self.lib, self.h)

    def density(self):
        rho = np.empty(self.n_atoms)
        _check(self.lib.dpd_get_density(self.h, capi.ptr(rho)), self.lib, self.h)
        return rho

    def cells(self):
        n = self.n_atoms
        cell = np.empty((n, 3), dtype=np.int32)
        off = np.empty((n, 3), dtype=np.float32)
        nc = np.empty(3, dtype=np.int32)
        w = np.empty(3, dtype=np.float32)
        cut2 = ctypes.c_float()
        _check(self.lib.dpd_get_cells(self.h, capi.ptr(cell), capi.ptr(off), capi.ptr(nc), capi.ptr(w),
                                      ctypes.byref(cut2)), self.lib, self.h)
        return {"cell": cell, "offset": off, "nc": nc, "w": w, "cut2": np.float32(cut2.value)}

    def neighbors(self):
        total = ctypes.c_int64()
        _check(self.lib.dpd_get_neighbors(self.h, None, 0, ctypes.byref(total)), self.lib, self.h)
        pairs = np.empty((max(total.value, 1), 2), dtype=np.int32)
        _check(self.lib.dpd_get_neighbors(self.h, capi.ptr(pairs), total.value, ctypes.byref(total)),
               self.lib, self.h)
        return pairs[: total.value]

    def rdf(self, nbins):
        g = np.empty(nbins)
        ns = ctypes.c_int64()
        _check(self.lib.dpd_rdf_result(self.h, capi.ptr(g), ctypes.byref(ns)), self.lib, self.h)
        return g, ns.value

    def info(self):
        st, nb, na, db = (ctypes.c_int64() for _ in range(4))
        _check(self.lib.dpd_get_info(self.h, ctypes.byref(st), ctypes.byref(nb), ctypes.byref(na),
                                     ctypes.byref(db)), self.lib, self.h)
        return {"step": st.value, "builds": nb.value, "atoms": na.value, "device_bytes": db.value}

    def time_steps(self, nsteps):
        tot, pair, nl = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        _check(self.lib.dpd_time_steps(self.h, int(nsteps), ctypes.byref(tot), ctypes.byref(pair),
                                       ctypes.byref(nl)), self.lib, self.h)
        return {"total_ms": tot.value, "pair_ms": pair.value, "pair_launches": nl.value}

    def list_stats(self):
        p, n, b = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _check(self.lib.dpd_get_list_stats(self.h, ctypes.byref(p), ctypes.byref(n), ctypes.byref(b)),
               self.lib, self.h)
        return {"pairs": p.value, "atoms": n.value, "builds": b.value,
                "mean_half_list": p.value / max(n.value, 1)}

    def write_data(self, path):
        _check(self.lib.dpd_write_data(self.h, path.encode()), self.lib, self.h)

    def bond_compute_aos(self, d_pos, d_bondlist, n_bonds, d_force, d_bond_pe=None, d_virial=None):
        """Bond::compute_force on AoS device buffers (integer device addresses)."""
        _check(self.lib.dpd_bond_compute_aos(self.h, d_pos, d_bondlist, int(n_bonds), d_force, d_bond_pe, d_virial),
               self.lib, self.h)

    def nve_aos(self, phase, d_group, n_group, d_type, d_pos, d_uwpos, d_vel, d_force):
        """fix nve's initial (phase 0) or final (phase 1) step on AoS device buffers."""
        _check(self.lib.dpd_nve_aos(self.h, int(phase), d_group, int(n_group), d_type, d_pos, d_uwpos, d_vel,
                                    d_force), self.lib, self.h)

    def pair_compute_aos(self, d_pos, d_vel, d_id, d_type, n, step, d_force, d_pe=None, d_virial=None):
        """Pair::compute_force on AoS device buffers (integer device addresses)."""
        _check(self.lib.dpd_pair_compute_aos(self.h, d_pos, d_vel, d_id, d_type, int(n), int(step), d_force,
                                             d_pe, d_virial), self.lib, self.h)

    def set_tuning(self, **knobs):
        """Launch knobs (the fields of dpd_tuning); those not named take the engine defaults
        (capi.DEFAULT_TUNING, zero for the rest)."""
        t = capi.tuning(**knobs)
        _check(self.lib.dpd_set_tuning(self.h, ctypes.byref(t)), self.lib, self.h)


class Batch:
    """Many independent systems advanced together in one packed engine."""

    def __init__(self, run_ins, systems, tuning=None):
        self.lib = capi.load()
        self.h = ctypes.c_void_p()
        n = len(run_ins)
        texts = (ctypes.c_char_p * n)(*[t.encode() for t in run_ins])
        structs = (capi.dpd_system * n)()
        self._keep = [texts]
        self.n_atoms = []
        for r, (s, keep) in enumerate(systems):
            structs[r] = s
            self._keep.append(keep)
            self.n_atoms.append(s.n_atoms)
        self._keep.append(structs)
        tune = None
        if tuning is not None:
            tune = capi.tuning(**tuning)
            self._keep.append(tune)
            tune = ctypes.byref(tune)
        code = self.lib.dpd_batch_create(n, texts, structs, tune, ctypes.byref(self.h))
        _check(code, self.lib, None)
        self.n = n

    def close(self):
        if self.h:
            self.lib.dpd_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, nsteps):
        _check(self.lib.dpd_run(self.h, int(nsteps)), self.lib, self.h)

    def set_tuning(self, **knobs):
        """Launch knobs (the fields of dpd_tuning); those not named take the engine defaults
        (capi.DEFAULT_TUNING, zero for the rest)."""
        t = capi.tuning(**knobs)
        _check(self.lib.dpd_set_tuning(self.h, ctypes.byref(t)), self.lib, self.h)

    def thermo(self, rep, max_rows=4096):
        rows = (capi.dpd_thermo * max_rows)()
        n = ctypes.c_int()
        _check(self.lib.dpd_batch_get_thermo(self.h, rep, rows, max_rows, ctypes.byref(n)), self.lib, self.h)
        return _rows_to_dict(rows, n.value)

    def state(self, rep):
        n = self.n_atoms[rep]
        x, v, f = np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
        img = np.empty((n, 3), dtype=np.int32)
        _check(self.lib.dpd_batch_get_state(self.h, rep, capi.ptr(x), capi.ptr(v), capi.ptr(img), capi.ptr(f)),
               self.lib, self.h)
        return {"x": x, "v": v, "image": img, "f": f}

    def rdf(self, rep, nbins):
        g = np.empty(nbins)
        ns = ctypes.c_int64()
        _check(self.lib.dpd_batch_rdf_result(self.h, rep, capi.ptr(g), ctypes.byref(ns)), self.lib, self.h)
        return g, ns.value

    def time_steps(self, nsteps):
        tot, pair, nl = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        _check(self.lib.dpd_time_steps(self.h, int(nsteps), ctypes.byref(tot), ctypes.byref(pair),
                                       ctypes.byref(nl)), self.lib, self.h)
        return {"total_ms": tot.value, "pair_ms": pair.value, "pair_launches": nl.value}
