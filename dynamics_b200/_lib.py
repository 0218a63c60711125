"""ctypes binding of libdynb200.so (the C ABI in include/dynb200.h).

The library is loaded from this package directory only; there is no other
implementation of the engine, so a missing library raises instead of
falling back to anything.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdynb200.so")

DYN_OK = 0
DYN_ERR_INVALID = -1
DYN_ERR_CUDA = -2
DYN_ERR_OOM = -3
DYN_ERR_NONFINITE = -5
DYN_ERR_TIMEOUT = -6
DYN_ERR_UNSUPPORTED = -7

DYN_NB_STATIC_MAX_SITES = 131072
DYN_STAGES = 13
DYN_OVR_COULOMB_DISABLED = 1
DYN_OVR_LJ_DISABLED = 2
DYN_PAIR_SCALE14 = 1
DYN_PAIR_LJ = 2
DYN_PAIR_COULOMB = 4
DYN_PAIR_SYMMETRIC = 8
DYN_PAIR_ALCH = 16

DYN_INTEGRATOR_LANGEVIN_MIDDLE = 0
DYN_INTEGRATOR_VERLET_VELOCITY = 1
DYN_THERMO_NONE = 0
DYN_THERMO_CSVR = 1
DYN_BARO_NONE = 0
DYN_BARO_CRESCALE = 1
DYN_FLAG_EWALD_CORRECTIONS = 1
DYN_FLAG_FULL_ENERGY = 2
DYN_FLAG_COM_REMOVAL = 4
DYN_FLAG_RECENTER = 8
DYN_FLAG_RESET_ANGLE = 16
DYN_FLAG_RATTLE_VELOCITIES = 32


class DynError(RuntimeError):
    """A dynb200 call returned a non-zero status."""

    def __init__(self, code, msg):
        super().__init__(f"dynb200 error {code}: {msg}")
        self.code = code


class Config(C.Structure):
    _fields_ = [
        ("box_lo", C.c_float * 3), ("box_hi", C.c_float * 3),
        ("coulomb_cutoff", C.c_float), ("lj_cutoff", C.c_float), ("list_buffer", C.c_float),
        ("ewald_alpha", C.c_float), ("grid", C.c_uint32 * 3),
        ("integrator", C.c_uint32), ("thermostat", C.c_uint32), ("barostat", C.c_uint32),
        ("temperature", C.c_float), ("langevin_gamma", C.c_float), ("tau_temp", C.c_float),
        ("pressure_bar", C.c_float), ("tau_pressure", C.c_float), ("compressibility", C.c_float),
        ("spme_interval", C.c_uint32), ("com_interval", C.c_uint32),
        ("recenter_interval", C.c_uint32), ("energy_interval", C.c_uint32),
        ("flags", C.c_uint32), ("thermo_dof", C.c_uint32), ("seed", C.c_uint64),
        ("ww_union_chunk", C.c_uint32), ("lincs_order", C.c_uint32), ("lincs_iter", C.c_uint32),
        ("prune_buffer", C.c_float),
        ("alch_begin", C.c_uint32), ("alch_end", C.c_uint32), ("alch_lambda", C.c_float),
        ("spme_brick_cap", C.c_uint32), ("pair_item_entries", C.c_uint32), ("ww_split", C.c_uint32),
    ]


_P = C.c_void_p


class SystemDesc(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_uint32), ("atom_pos", _P), ("atom_vel", _P), ("atom_mass", _P),
        ("atom_q", _P), ("atom_sigma", _P), ("atom_eps", _P), ("atom_static", _P),
        ("n_water", C.c_uint32), ("water_pos", _P), ("water_vel", _P),
        ("n_excl", C.c_uint32), ("excl", _P),
        ("n_pair14", C.c_uint32), ("pair14", _P),
        ("n_bonds", C.c_uint32), ("bonds", _P), ("bond_k", _P), ("bond_r0", _P),
        ("n_angles", C.c_uint32), ("angles", _P), ("angle_k", _P), ("angle_theta0", _P),
        ("n_dihedrals", C.c_uint32), ("dihedrals", _P), ("dihedral_k", _P), ("dihedral_n", _P),
        ("dihedral_phase", _P),
        ("n_constraints", C.c_uint32), ("constraints", _P), ("constraint_r0", _P),
    ]


class Energies(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "kinetic", "kinetic_trans", "potential", "e_lj", "e_coul_short", "e_water_water_short",
        "e_recip", "e_corrections", "e_bonded", "virial", "virial_short", "virial_recip",
        "virial_bonded", "virial_constraints", "pressure_bar", "temperature")] + [
        ("box", C.c_double * 3), ("step", C.c_uint64), ("list_rebuilds", C.c_uint64),
        ("pairs_in_list", C.c_uint64), ("kinetic_rigid", C.c_double),
        ("pressure_atomic_bar", C.c_double), ("list_union_max", C.c_uint64), ("dh_dl", C.c_double),
        ("list_prunes", C.c_uint64)]

    def as_dict(self):
        d = {n: getattr(self, n) for n, _ in self._fields_ if n != "box"}
        d["box"] = [self.box[i] for i in range(3)]
        return d


class Frame(C.Structure):
    """dyn_frame_t: one snapshot frame's scalars."""
    _fields_ = [("step", C.c_uint64)] + [(n, C.c_double) for n in (
        "time_ps", "kinetic", "potential", "potential_bonded", "temperature", "pressure_bar")] + [
        ("box_lo", C.c_double * 3), ("box_hi", C.c_double * 3), ("volume", C.c_double),
        ("density", C.c_double), ("dh_dl", C.c_double)]

    def as_dict(self):
        d = {n: getattr(self, n) for n, _ in self._fields_ if n not in ("box_lo", "box_hi")}
        d["box_lo"] = [self.box_lo[i] for i in range(3)]
        d["box_hi"] = [self.box_hi[i] for i in range(3)]
        return d


DYN_SNAP_VELOCITIES = 1
DYN_SNAP_FORCES = 2

_lib = None

_SIGS = {
    "dyn_last_error": ([], C.c_char_p),
    "dyn_version": ([], C.c_int),
    "dyn_device_count": ([], C.c_int),
    "dyn_probe_fp32_peak": ([_P, _P], C.c_int),
    "dyn_nb_create": ([_P, C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_float, _P], C.c_int),
    "dyn_nb_set_pairs": ([_P, C.c_uint64] + [_P] * 9, C.c_int),
    "dyn_nb_build_pairs": ([_P, _P, _P, _P, _P, _P, _P, _P, C.c_uint64, _P, C.c_uint64, _P, _P, _P,
                            C.c_float, _P], C.c_int),
    "dyn_nb_get_pairs": ([_P, C.c_uint64] + [_P] * 9, C.c_int),
    "dyn_nb_forces": ([_P, _P, _P, _P, _P, _P, _P, C.c_uint32, _P, _P, _P, _P, _P, _P, _P], C.c_int),
    "dyn_nb_forces_alch": ([_P, _P, _P, _P, _P, _P, _P, C.c_uint32, C.c_double]
                           + [_P] * 8, C.c_int),
    "dyn_nb_mark_alch": ([_P, C.c_uint32, C.c_uint32, _P], C.c_int),
    "dyn_nb_forces_static": ([_P, C.c_uint32, C.c_uint32, _P, _P, _P, _P, _P, C.c_uint64]
                             + [_P] * 9 + [_P, C.c_float, C.c_float, C.c_float, C.c_uint32]
                             + [_P] * 6, C.c_int),
    "dyn_nb_destroy": ([_P], C.c_int),
    "dyn_sys_create": ([_P, _P, _P, _P], C.c_int),
    "dyn_sys_step": ([_P, C.c_uint32, C.c_float], C.c_int),
    "dyn_sys_forces": ([_P, _P, _P, _P], C.c_int),
    "dyn_sys_get_state": ([_P, _P, _P, _P, _P, _P], C.c_int),
    "dyn_sys_set_state": ([_P, _P, _P, _P, _P], C.c_int),
    "dyn_sys_get_energies": ([_P, _P], C.c_int),
    "dyn_sys_sync": ([_P], C.c_int),
    "dyn_sys_destroy": ([_P], C.c_int),
    "dyn_sys_step_host": ([_P, C.c_uint32, C.c_float] + [_P] * 9, C.c_int),
    "dyn_sys_stage_times": ([_P, C.c_uint32, C.c_float, _P], C.c_int),
    "dyn_sys_launches_per_step": ([_P, C.c_int, _P], C.c_int),
    "dyn_sys_launches_conditional": ([_P, _P, _P], C.c_int),
    "dyn_batch_create": ([_P, C.c_uint32, _P, _P, _P], C.c_int),
    "dyn_batch_step": ([_P, C.c_uint32, C.c_float], C.c_int),
    "dyn_batch_size": ([_P, _P], C.c_int),
    "dyn_batch_member": ([_P, C.c_uint32, _P], C.c_int),
    "dyn_batch_sync": ([_P], C.c_int),
    "dyn_batch_launches": ([_P, C.c_int, _P, _P, _P], C.c_int),
    "dyn_batch_destroy": ([_P], C.c_int),
    "dyn_batch_add": ([_P, _P, _P, _P], C.c_int),
    "dyn_batch_remove": ([_P, C.c_uint32], C.c_int),
    "dyn_batch_memory": ([_P, _P], C.c_int),
    "dyn_batch_state_layout": ([_P, _P], C.c_int),
    "dyn_batch_host_buffer": ([_P, _P, _P], C.c_int),
    "dyn_batch_step_host": ([_P, C.c_uint32, C.c_float, _P, _P, _P], C.c_int),
    "dyn_sys_memory": ([_P, _P], C.c_int),
    "dyn_sys_snapshots": ([_P, C.c_uint32, C.c_uint32, C.c_uint32], C.c_int),
    "dyn_sys_minimize": ([_P, C.c_uint32, C.c_float, _P, _P], C.c_int),
    "dyn_sys_set_static": ([_P, _P, C.c_uint32], C.c_int),
    "dyn_sys_set_lambda": ([_P, C.c_float], C.c_int),
    "dyn_sys_snapshots_read": ([_P, C.c_uint32, _P, _P, _P, _P, _P, _P], C.c_int),
    "dyn_sys_list_pairs": ([_P, C.c_uint32, _P, C.c_uint64, _P], C.c_int),
}

EXPORTED = tuple(_SIGS)


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise DynError(DYN_ERR_UNSUPPORTED,
                           f"{LIB_PATH} is missing; run `python -m dynamics_b200.build`")
        l = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            f = getattr(l, name)
            f.argtypes = args
            f.restype = res
        _lib = l
    return _lib


def check(code):
    if code != DYN_OK:
        raise DynError(code, lib().dyn_last_error().decode())
    return code


def ptr(a):
    """Address of a contiguous numpy array (None -> NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def f32(a, n=None):
    x = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    if n is not None:
        x = x.reshape(n)
    return x


def u32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def u8(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint8))
