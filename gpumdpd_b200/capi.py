"""ctypes binding of libdpd_b200.so (declared in include/dpd_b200.h).

The library is built in-tree (``make -C gpumdpd_b200``).  Loading fails loudly when
it is missing: the engine has no CPU fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdpd_b200.so")

DPD_ERRORS = {
    -1: "DPD_E_ARG", -2: "DPD_E_IO", -3: "DPD_E_CUDA", -4: "DPD_E_NOMEM",
    -5: "DPD_E_OVERFLOW", -6: "DPD_E_STATE", -7: "DPD_E_NUMERIC", -8: "DPD_E_NODEV",
    -9: "DPD_E_CANCELLED",
}

# every symbol declared in include/dpd_b200.h
EXPORTED = [
    "dpd_create", "dpd_create_from_system", "dpd_create_fp64", "dpd_run", "dpd_sync", "dpd_get_thermo", "dpd_get_spring_records",
    "dpd_dump_open", "dpd_compute_dump_open", "dpd_dump_close", "dpd_bond_compute_aos", "dpd_nve_aos", "dpd_write_restart", "dpd_read_restart", "dpd_get_compute",
    "dpd_get_state", "dpd_set_state", "dpd_get_density", "dpd_get_cells", "dpd_get_neighbors",
    "dpd_compute_rdf", "dpd_rdf_config", "dpd_rdf_result", "dpd_get_info", "dpd_set_tuning",
    "dpd_write_data", "dpd_time_steps", "dpd_get_list_stats", "dpd_last_error", "dpd_destroy", "dpd_pair_compute_aos",
    "dpd_batch_create", "dpd_batch_n", "dpd_batch_get_thermo", "dpd_batch_get_state",
    "dpd_batch_rdf_result", "dpd_server_create", "dpd_server_submit", "dpd_server_set_policy", "dpd_server_step",
    "dpd_server_result", "dpd_server_cancel", "dpd_server_job_state", "dpd_server_job_rdf", "dpd_server_stats",
    "dpd_server_last_error", "dpd_server_destroy", "dpd_pair_forces_noalloc", "dpd_version",
]

NOALLOC_MAX_ATOMS = 262144
NOALLOC_MAX_CELLS = 262144
NOALLOC_MAX_TYPES = 8


class DpdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{DPD_ERRORS.get(code, code)}: {msg}")
        self.code = code


class dpd_system(ctypes.Structure):
    _fields_ = [
        ("n_atoms", ctypes.c_int), ("n_atomtypes", ctypes.c_int), ("n_bonds", ctypes.c_int),
        ("n_bondtypes", ctypes.c_int), ("lo", ctypes.c_double * 3), ("hi", ctypes.c_double * 3),
        ("masses", ctypes.POINTER(ctypes.c_double)), ("tag", ctypes.POINTER(ctypes.c_int)),
        ("type", ctypes.POINTER(ctypes.c_int)), ("mol", ctypes.POINTER(ctypes.c_int)),
        ("x", ctypes.POINTER(ctypes.c_double)), ("v", ctypes.POINTER(ctypes.c_double)),
        ("bonds", ctypes.POINTER(ctypes.c_int)),
        ("n_angles", ctypes.c_int), ("n_angletypes", ctypes.c_int),
        ("angles", ctypes.POINTER(ctypes.c_int)),
    ]


class dpd_thermo(ctypes.Structure):
    _fields_ = [
        ("step", ctypes.c_int64), ("temp", ctypes.c_double), ("pair_pe", ctypes.c_double),
        ("bond_pe", ctypes.c_double), ("pressure", ctypes.c_double), ("p", ctypes.c_double * 6),
        ("ke", ctypes.c_double), ("momentum", ctypes.c_double * 3),
        ("angle_pe", ctypes.c_double),
    ]


class dpd_tuning(ctypes.Structure):
    _fields_ = [
        ("pair_block", ctypes.c_int), ("pair_variant", ctypes.c_int), ("cell_order", ctypes.c_int),
        ("build_variant", ctypes.c_int), ("launch_mode", ctypes.c_int), ("tile", ctypes.c_int),
        ("tile_capacity", ctypes.c_int), ("reserved", ctypes.c_int),
    ]


# the engine's knobs when none are given (pair schedule 8, linear cells, column-range build)
DEFAULT_TUNING = {"pair_variant": 8, "cell_order": 0, "build_variant": 5}


def tuning(**knobs):
    """A dpd_tuning of the engine defaults with the given knobs replaced."""
    t = dpd_tuning()
    for k, v in {**DEFAULT_TUNING, **knobs}.items():
        if not hasattr(t, k) or k == "reserved":
            raise TypeError(f"unknown tuning knob {k!r}")
        setattr(t, k, int(v))
    return t


class dpd_job_result(ctypes.Structure):
    _fields_ = [
        ("job_id", ctypes.c_int64), ("status", ctypes.c_int), ("steps", ctypes.c_int64),
        ("mean_temp", ctypes.c_double), ("mean_pressure", ctypes.c_double),
        ("submit_s", ctypes.c_double), ("start_s", ctypes.c_double), ("finish_s", ctypes.c_double),
        ("last", dpd_thermo),
        ("stderr_temp", ctypes.c_double), ("stderr_pressure", ctypes.c_double),
    ]


class dpd_pair_params(ctypes.Structure):
    _fields_ = [
        ("lo", ctypes.c_double * 3), ("hi", ctypes.c_double * 3), ("ntypes", ctypes.c_int),
        ("coeff", ((ctypes.c_double * 3) * NOALLOC_MAX_TYPES) * NOALLOC_MAX_TYPES),
        ("kT", ctypes.c_double), ("dt", ctypes.c_double), ("seed", ctypes.c_uint32),
    ]


_lib = None


def load():
    """Load libdpd_b200.so (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `make -C {_HERE}` "
                          "(the engine has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    i, i64, u32, d, cp = ctypes.c_int, ctypes.c_int64, ctypes.c_uint32, ctypes.c_double, ctypes.c_char_p
    sig = {
        "dpd_create": (i, [cp, cp, cp, P(vp)]),
        "dpd_create_from_system": (i, [cp, P(dpd_system), P(vp)]),
        "dpd_create_fp64": (i, [cp, cp, cp, P(dpd_system), P(vp)]),
        "dpd_run": (i, [vp, u32]),
        "dpd_sync": (i, [vp]),
        "dpd_get_thermo": (i, [vp, P(dpd_thermo), i, P(i)]),
        "dpd_get_spring_records": (i, [vp, vp, i, P(i)]),
        "dpd_dump_open": (i, [vp, cp, i64, i64, i]),
        "dpd_dump_close": (i, [vp]),
        "dpd_bond_compute_aos": (i, [vp, vp, vp, i, vp, vp, vp]),
        "dpd_nve_aos": (i, [vp, i, vp, i, vp, vp, vp, vp, vp]),
        "dpd_compute_dump_open": (i, [vp, cp, cp]),
        "dpd_write_restart": (i, [vp, cp]),
        "dpd_get_compute": (i, [vp, cp, vp, i, P(i), P(i)]),
        "dpd_read_restart": (i, [vp, cp]),
        "dpd_get_state": (i, [vp, vp, vp, vp, vp]),
        "dpd_set_state": (i, [vp, vp, vp]),
        "dpd_get_density": (i, [vp, vp]),
        "dpd_get_cells": (i, [vp, vp, vp, vp, vp, vp]),
        "dpd_get_neighbors": (i, [vp, vp, i64, P(i64)]),
        "dpd_compute_rdf": (i, [vp, i, i, d, i, vp]),
        "dpd_rdf_config": (i, [vp, i, i, d, i, i]),
        "dpd_rdf_result": (i, [vp, vp, P(i64)]),
        "dpd_get_info": (i, [vp, P(i64), P(i64), P(i64), P(i64)]),
        "dpd_set_tuning": (i, [vp, P(dpd_tuning)]),
        "dpd_get_list_stats": (i, [vp, P(i64), P(i64), P(i64)]),
        "dpd_write_data": (i, [vp, cp]),
        "dpd_time_steps": (i, [vp, u32, P(d), P(d), P(i64)]),
        "dpd_last_error": (cp, [vp]),
        "dpd_destroy": (i, [vp]),
        "dpd_pair_compute_aos": (i, [vp, vp, vp, vp, vp, i, u32, vp, vp, vp]),
        "dpd_batch_create": (i, [i, P(cp), P(dpd_system), P(dpd_tuning), P(vp)]),
        "dpd_batch_n": (i, [vp, P(i)]),
        "dpd_batch_get_thermo": (i, [vp, i, P(dpd_thermo), i, P(i)]),
        "dpd_batch_get_state": (i, [vp, i, vp, vp, vp, vp]),
        "dpd_batch_rdf_result": (i, [vp, i, vp, P(i64)]),
        "dpd_server_create": (i, [d, i, P(dpd_tuning), P(vp)]),
        "dpd_server_submit": (i, [vp, cp, P(dpd_system), P(i64)]),
        "dpd_server_set_policy": (i, [vp, d, i]),
        "dpd_server_step": (i, [vp, P(i), P(i)]),
        "dpd_server_result": (i, [vp, i64, P(dpd_job_result)]),
        "dpd_server_cancel": (i, [vp, i64]),
        "dpd_server_job_state": (i, [vp, i64, vp, vp]),
        "dpd_server_job_rdf": (i, [vp, i64, vp, P(i64)]),
        "dpd_server_stats": (i, [vp, P(i64), P(d), P(i64)]),
        "dpd_server_last_error": (cp, [vp]),
        "dpd_server_destroy": (i, [vp]),
        "dpd_pair_forces_noalloc": (i, [P(dpd_pair_params), vp, vp, vp, vp, i, u32, vp, vp]),
        "dpd_version": (cp, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(a):
    """ctypes void pointer of a contiguous numpy array (or None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def make_system(box_lo, box_hi, masses, types, x, v=None, bonds=None, n_bondtypes=0, mol=None,
                tags=None, angles=None, n_angletypes=0):
    """Build a dpd_system from numpy arrays; returns (struct, keepalive list)."""
    n = len(types)
    masses = np.ascontiguousarray(masses, dtype=np.float64)
    types = np.ascontiguousarray(types, dtype=np.int32)
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    tags = np.arange(1, n + 1, dtype=np.int32) if tags is None else np.ascontiguousarray(tags, dtype=np.int32)
    keep = [masses, types, x, tags]
    s = dpd_system()
    s.n_atoms = n
    s.n_atomtypes = len(masses)
    s.lo = (ctypes.c_double * 3)(*box_lo)
    s.hi = (ctypes.c_double * 3)(*box_hi)
    s.masses = masses.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    s.tag = tags.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    s.type = types.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    s.x = x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    if v is not None:
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        keep.append(v)
        s.v = v.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    if mol is not None:
        mol = np.ascontiguousarray(mol, dtype=np.int32)
        keep.append(mol)
        s.mol = mol.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    if bonds is not None and len(bonds):
        bonds = np.ascontiguousarray(bonds, dtype=np.int32).reshape(-1)
        keep.append(bonds)
        s.n_bonds = len(bonds) // 3
        s.n_bondtypes = max(int(n_bondtypes), 1)
        s.bonds = bonds.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    else:
        s.n_bonds = 0
        s.n_bondtypes = int(n_bondtypes)
    if angles is not None and len(angles):
        angles = np.ascontiguousarray(angles, dtype=np.int32).reshape(-1)
        keep.append(angles)
        s.n_angles = len(angles) // 4
        s.n_angletypes = max(int(n_angletypes), 1)
        s.angles = angles.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    else:
        s.n_angles = 0
        s.n_angletypes = int(n_angletypes)
    return s, keep
