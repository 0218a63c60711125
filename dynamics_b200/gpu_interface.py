"""Python mirror of the reference's GPU boundary, src/gpu_interface.rs.

Same names and argument meaning as the Rust module, backed by the C ABI
(dyn_nb_*), so code written against the reference's boundary ports over
line by line:

    ForcesPositsGpu::new(stream, n_dyn, n_water, cutoff_ewald, alpha_ewald)
        -> ForcesPositsGpu(n_dyn, n_water, cutoff_ewald, alpha_ewald)
    PerNeighborGpu::new(stream, pairs, atoms_dyn, water, lj_tables)
        -> PerNeighborGpu(forces, pairs)             (flat pair SoA dict)
    build_all_neighbors + setup_pairs + PerNeighborGpu::new
        -> PerNeighborGpu.build(forces, ...)          (on the GPU)
    force_nonbonded_gpu(stream, kernels, pairs, atoms_dyn, water, cell_extent,
                        forces, per_neighbor, overrides, lambda_alch)
        -> force_nonbonded_gpu(forces, per_neighbor, pos_dyn, pos_water,
                               cell_extent, overrides, lambda_alch)
    setup_pairs' alch_interaction for molecule m (atoms [b, e))
        -> PerNeighborGpu.mark_alchemical(b, e), or the ``alch`` column

Errors raise DynError instead of panicking or printing (the reference
unwraps and eprintln!s, src/gpu_interface.rs:557-564).
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, f32, lib, ptr, u8, u32

BODY_ATOM, BODY_W_O, BODY_W_M, BODY_W_H0, BODY_W_H1 = 0, 1, 2, 3, 4


class ForcesPositsGpu:
    """Device and pinned buffers for one system (src/gpu_interface.rs:84-215).

    ``lj_cutoff <= 0`` reproduces the reference CUDA kernel (no LJ cutoff);
    ``lj_cutoff > 0`` reproduces the reference CPU path (LJ for r <= lj_cutoff).
    """

    def __init__(self, n_dyn, n_water, cutoff_ewald, alpha_ewald, lj_cutoff=0.0, stream=None):
        h = C.c_void_p()
        check(lib().dyn_nb_create(stream, int(n_dyn), int(n_water), float(cutoff_ewald),
                                  float(alpha_ewald), float(lj_cutoff), C.byref(h)))
        self._h = h
        self.n_dyn = int(n_dyn)
        self.n_water = int(n_water)

    @property
    def handle(self):
        if self._h is None:
            raise _lib.DynError(_lib.DYN_ERR_INVALID, "ForcesPositsGpu already closed")
        return self._h

    def close(self):
        if self._h is not None:
            lib().dyn_nb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pack_flags(pairs):
    fl = np.zeros(len(pairs["tgt"]), dtype=np.uint8)
    fl |= np.asarray(pairs["scale_14"], dtype=np.uint8) * _lib.DYN_PAIR_SCALE14
    fl |= np.asarray(pairs["calc_lj"], dtype=np.uint8) * _lib.DYN_PAIR_LJ
    fl |= np.asarray(pairs["calc_coulomb"], dtype=np.uint8) * _lib.DYN_PAIR_COULOMB
    fl |= np.asarray(pairs["symmetric"], dtype=np.uint8) * _lib.DYN_PAIR_SYMMETRIC
    if "alch" in pairs:
        fl |= np.asarray(pairs["alch"], dtype=np.uint8) * _lib.DYN_PAIR_ALCH
    return fl


class PerNeighborGpu:
    """Per-pair metadata on the device (src/gpu_interface.rs:222-411).

    ``pairs`` is the flat SoA the reference builds: tgt, src (uint32), sigma,
    eps, q_tgt, q_src (float32), body_tgt / body_src (0 atom, 1..4 water
    O, M, H0, H1) and the bool arrays scale_14, calc_lj, calc_coulomb,
    symmetric and, optionally, alch (alch_interaction).  (The reference's atom_types_* + water_types_* pair maps onto
    body_* as body = water_type for water ends and 0 otherwise.)
    """

    def __init__(self, forces, pairs=None):
        self.forces = forces
        self.n_pairs = 0
        if pairs is not None:
            self.set_pairs(pairs)

    def set_pairs(self, pairs):
        n = len(pairs["tgt"])
        bt = pairs.get("body_tgt")
        bs = pairs.get("body_src")
        if bt is None:
            bt = np.where(np.asarray(pairs["atype_tgt"]) == 0, 0, pairs["wtype_tgt"])
            bs = np.where(np.asarray(pairs["atype_src"]) == 0, 0, pairs["wtype_src"])
        arrs = [u32(pairs["tgt"]), u32(pairs["src"]), f32(pairs["sigma"]), f32(pairs["eps"]),
                f32(pairs["q_tgt"]), f32(pairs["q_src"]), u8(bt), u8(bs), pack_flags(pairs)]
        check(lib().dyn_nb_set_pairs(self.forces.handle, n, *[ptr(a) for a in arrs]))
        self.n_pairs = n

    @classmethod
    def build(cls, forces, pos_dyn, pos_w_o, atom_q, atom_sigma, atom_eps, box_lo, box_hi, skin,
              excl=None, pair14=None, is_static=None, bonded_only=None):
        """build_all_neighbors + setup_pairs on the GPU (bit-exact pair set)."""
        self = cls(forces)
        nd = forces.n_dyn
        pd = f32(pos_dyn).reshape(-1) if nd else None
        po = f32(pos_w_o).reshape(-1) if forces.n_water else None
        q = f32(atom_q) if nd else None
        sg = f32(atom_sigma) if nd else None
        ep = f32(atom_eps) if nd else None
        st = u8(is_static) if is_static is not None else None
        bo = u8(bonded_only) if bonded_only is not None else None
        ex = u32(excl).reshape(-1) if excl is not None and len(excl) else None
        p14 = u32(pair14).reshape(-1) if pair14 is not None and len(pair14) else None
        lo = f32(box_lo, 3)
        hi = f32(box_hi, 3)
        n = C.c_uint64()
        check(lib().dyn_nb_build_pairs(
            forces.handle, ptr(pd), ptr(po), ptr(q), ptr(sg), ptr(ep), ptr(st), ptr(bo),
            0 if ex is None else len(ex) // 2, ptr(ex), 0 if p14 is None else len(p14) // 2, ptr(p14),
            ptr(lo), ptr(hi), float(skin), C.byref(n)))
        self.n_pairs = n.value
        return self

    def mark_alchemical(self, atom_begin, atom_end):
        """Flags the pairs crossing the boundary of the alchemical molecule
        (atoms [atom_begin, atom_end)) as setup_pairs does
        (src/non_bonded.rs:581-612); returns the number flagged."""
        n = C.c_uint64()
        check(lib().dyn_nb_mark_alch(self.forces.handle, int(atom_begin), int(atom_end), C.byref(n)))
        return n.value

    def get_pairs(self):
        """The installed list: tgt, src, body_tgt, body_src, flags, sigma,
        eps and qq (= q_tgt * q_src as stored on the device)."""
        n = self.n_pairs
        out = {
            "tgt": np.zeros(n, np.uint32), "src": np.zeros(n, np.uint32),
            "sigma": np.zeros(n, np.float32), "eps": np.zeros(n, np.float32),
            "qq": np.zeros(n, np.float32), "q_one": np.zeros(n, np.float32),
            "body_tgt": np.zeros(n, np.uint8), "body_src": np.zeros(n, np.uint8),
            "flags": np.zeros(n, np.uint8),
        }
        check(lib().dyn_nb_get_pairs(self.forces.handle, n, ptr(out["tgt"]), ptr(out["src"]),
                                     ptr(out["sigma"]), ptr(out["eps"]), ptr(out["qq"]),
                                     ptr(out["q_one"]), ptr(out["body_tgt"]), ptr(out["body_src"]),
                                     ptr(out["flags"])))
        del out["q_one"]
        return out


def force_nonbonded_gpu(forces, per_neighbor, pos_dyn, pos_water, cell_extent, overrides=0,
                        lambda_alch=None):
    """force_nonbonded_gpu (src/gpu_interface.rs:463-632).

    pos_water: dict {1: O, 2: M, 3: H0, 4: H1} or a sequence (O, M, H0, H1)
    of (n_water, 3) arrays.  Returns (f_dyn (n,3), f_water dict {1..4: (n,3)},
    virial, energy) in float64; with ``lambda_alch`` given, a fifth element,
    the alchemical pairs' dH/dlambda (0 when none is installed).
    """
    del per_neighbor  # the handle owns the installed list
    nd, nw = forces.n_dyn, forces.n_water
    if isinstance(pos_water, dict):
        pw = [pos_water[k] for k in (1, 2, 3, 4)]
    else:
        pw = list(pos_water)
    pd = f32(pos_dyn).reshape(-1) if nd else np.zeros(3, np.float32)
    pws = [f32(p).reshape(-1) if nw else np.zeros(3, np.float32) for p in pw]
    ext = f32(cell_extent, 3)
    fd = np.zeros((max(nd, 1), 3))
    fw = [np.zeros((max(nw, 1), 3)) for _ in range(4)]
    vir = C.c_double()
    en = C.c_double()
    if lambda_alch is None:
        check(lib().dyn_nb_forces(forces.handle, ptr(pd), *[ptr(p) for p in pws], ptr(ext),
                                  int(overrides), ptr(fd), *[ptr(f) for f in fw], C.byref(vir),
                                  C.byref(en)))
        return fd[:nd], {k + 1: fw[k][:nw] for k in range(4)}, vir.value, en.value
    dh = C.c_double()
    check(lib().dyn_nb_forces_alch(forces.handle, ptr(pd), *[ptr(p) for p in pws], ptr(ext),
                                   int(overrides), float(lambda_alch), ptr(fd),
                                   *[ptr(f) for f in fw], C.byref(vir), C.byref(en), C.byref(dh)))
    return fd[:nd], {k + 1: fw[k][:nw] for k in range(4)}, vir.value, en.value, dh.value
