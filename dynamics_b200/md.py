"""Python mirror of the reference's public simulation API (MdState, MdConfig).

The reference drives a simulation with ``MdState::new(dev, &MdConfig, ..)``
and ``MdState::step(dev, dt, external_force)`` (src/lib.rs:711,
src/integrate.rs:72).  Here ``MdState(system, MdConfig)`` uploads a system
once and ``step(dt, n)`` advances it on the device through the C ABI
(dyn_sys_*); coordinates, velocities, lists and PME grids stay in HBM.

``system`` is a dict of numpy arrays (see dynamics_b200.synth):
  box_lo, box_hi (3,); water_pos, water_vel (n_water, 3, 3) [O, H0, H1];
  atom_pos, atom_vel (n, 3); atom_mass, atom_q, atom_sigma, atom_eps (n,);
  atom_static (n,) optional; excl, pair14 (m, 2); bonds (m, 2) + bond_k,
  bond_r0; angles (m, 3) + angle_k, angle_theta0; dihedrals (m, 4) +
  dihedral_k, dihedral_n, dihedral_phase.
"""
import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib
from ._lib import check, f32, lib, ptr, u8, u32


@dataclass
class LangevinMiddle:
    """Integrator::LangevinMiddle { gamma } (src/integrate.rs:43)."""
    gamma: float = 0.5  # LANGEVIN_GAMMA_DEFAULT, src/thermostat.rs:32


@dataclass
class VerletVelocity:
    """Integrator::VerletVelocity { thermostat } (src/integrate.rs:39);
    ``thermostat`` is the CSVR time constant in ps, or None."""
    thermostat: Optional[float] = 0.1  # TAU_TEMP_DEFAULT, src/thermostat.rs:27


@dataclass
class BarostatCfg:
    """BarostatCfg (src/barostat.rs:32-50): C-rescale."""
    pressure_target: float = 1.0
    tau: float = 5.0
    solvent_compressibility: float = 4.5e-5


@dataclass
class SnapshotEnergyData:
    """SnapshotEnergyData (src/snapshot.rs:61-93): the scalars of a frame
    (kcal/mol, K, bar, A^3, amu/A^3)."""
    energy_kinetic: float
    energy_potential: float
    energy_potential_nonbonded: float
    energy_potential_bonded: float
    temperature: float
    pressure: float
    dh_dl: Optional[float]
    volume: float
    density: float


@dataclass
class Snapshot:
    """Snapshot (src/snapshot.rs:124-175): time (ps), atom positions wrapped
    into the cell, water O / H0 / H1 positions, and, when recorded, atom and
    water-O velocities and atom forces; ``cell`` = (box_lo, box_hi)."""
    time: float
    step: int
    atom_posits: np.ndarray
    water_o_posits: np.ndarray
    water_h0_posits: np.ndarray
    water_h1_posits: np.ndarray
    energy_data: SnapshotEnergyData
    cell: tuple
    atom_velocities: Optional[np.ndarray] = None
    water_velocities: Optional[np.ndarray] = None
    force: Optional[np.ndarray] = None


@dataclass
class MdConfig:
    """The fields of MdConfig (src/config.rs:43-107) this engine uses.

    ``neighbor_skin`` is the Verlet buffer of the cluster lists (the
    reference's default of 4 A sizes its flat lists; the cluster lists need
    far less, and results do not depend on it).  ``spme_grid`` replaces
    ``spme_mesh_spacing``: the grid is given explicitly.
    """
    integrator: object = field(default_factory=LangevinMiddle)
    temp_target: float = 300.0
    coulomb_cutoff: float = 10.0
    lj_cutoff: float = 10.0
    neighbor_skin: float = 1.5
    spme_alpha: float = 0.26
    spme_grid: tuple = (32, 32, 32)
    barostat_cfg: Optional[BarostatCfg] = None
    zero_com_drift: bool = True
    com_removal_interval: int = 100
    recenter_sim_box: bool = True
    spme_interval: int = 2          # SPME_RATIO, src/lib.rs:208
    energy_interval: int = 1
    ewald_corrections: bool = False
    full_energy: bool = False
    reset_angle: bool = True
    seed: int = 0
    ww_union_chunk: int = 0         # 0 = automatic (tuning knob only)
    # inner buffer of the pruned water-water lists (A); 0 = automatic
    # (tuning knob only, results do not depend on it)
    prune_buffer: float = 0.0
    # charged sites per SPME grid brick before the overflow path; 0 =
    # automatic (results do not depend on it)
    spme_brick_cap: int = 0
    # list entries per work item of the water-atom and atom-atom pair
    # kernels (1..32); 0 = 8 (tuning knob only)
    pair_item_entries: int = 0
    # CTAs sharing one water group's list entries (1..8); 0 = automatic
    # (tuning knob only)
    ww_split: int = 0
    lincs_order: int = 4            # HydrogenConstraint::Linear { order, iter } (src/prep.rs:77)
    lincs_iter: int = 1
    # constraint position corrections also correct the velocities (RATTLE);
    # False = the reference's position-only correction, which dissipates
    # kinetic energy of the constrained bonds
    rattle_velocities: bool = False
    # alchemical decoupling of the atoms [begin, end) (one molecule) at
    # alch_lambda on the reference's staged schedule (src/alchemical.rs)
    alch_range: Optional[tuple] = None
    alch_lambda: float = 0.0
    # SnapshotHandlers.memory (src/snapshot.rs:34-46): record a snapshot
    # every this many steps into the device ring (None = off); the frames
    # come back through MdState.snapshots
    snapshot_memory: Optional[int] = None
    snapshot_capacity: int = 256


def thermo_dof(system, cfg):
    """dof_for_thermo (src/thermostat.rs:220-251): 6 per water, 3 per
    non-static atom, minus 3 with COM removal.  The reference subtracts the
    constrained hydrogens only for its SHAKE constraints, not for the
    default LINCS-style ones; here they are subtracted (non-static ones)
    with the RATTLE option, the constrained integrator that holds them."""
    nw = len(np.asarray(system.get("water_pos", np.zeros((0, 3, 3)))).reshape(-1, 3, 3))
    na = len(np.asarray(system.get("atom_pos", np.zeros((0, 3)))).reshape(-1, 3))
    st = np.asarray(system.get("atom_static", np.zeros(na, bool)), dtype=bool)
    dof = 6 * nw + 3 * int(np.count_nonzero(~st))
    if getattr(cfg, "rattle_velocities", False):
        cons = np.asarray(system.get("constraints", np.zeros((0, 2))), np.int64).reshape(-1, 2)
        if len(cons):
            dof -= int(np.count_nonzero(~st[cons[:, 1]]))
    if cfg.zero_com_drift:
        dof -= 3
    return max(dof, 0)


def _config_struct(system, cfg):
    c = _lib.Config()
    lo = f32(system["box_lo"], 3)
    hi = f32(system["box_hi"], 3)
    for k in range(3):
        c.box_lo[k] = lo[k]
        c.box_hi[k] = hi[k]
        c.grid[k] = int(cfg.spme_grid[k])
    c.coulomb_cutoff = cfg.coulomb_cutoff
    c.lj_cutoff = cfg.lj_cutoff
    c.list_buffer = cfg.neighbor_skin
    c.ewald_alpha = cfg.spme_alpha
    integ = cfg.integrator
    if isinstance(integ, LangevinMiddle):
        c.integrator = _lib.DYN_INTEGRATOR_LANGEVIN_MIDDLE
        c.langevin_gamma = integ.gamma
    elif isinstance(integ, VerletVelocity):
        c.integrator = _lib.DYN_INTEGRATOR_VERLET_VELOCITY
        c.thermostat = _lib.DYN_THERMO_CSVR if integ.thermostat else _lib.DYN_THERMO_NONE
        c.tau_temp = float(integ.thermostat or 0.0)
    else:
        raise _lib.DynError(_lib.DYN_ERR_INVALID, f"unsupported integrator {integ!r}")
    if cfg.barostat_cfg is not None:
        c.barostat = _lib.DYN_BARO_CRESCALE
        c.pressure_bar = cfg.barostat_cfg.pressure_target
        c.tau_pressure = cfg.barostat_cfg.tau
        c.compressibility = cfg.barostat_cfg.solvent_compressibility
    c.temperature = cfg.temp_target
    c.spme_interval = max(1, int(cfg.spme_interval))
    c.com_interval = int(cfg.com_removal_interval)
    c.recenter_interval = 30  # CENTER_SIMBOX_RATIO, src/lib.rs:204
    c.energy_interval = max(1, int(cfg.energy_interval))
    flags = 0
    if cfg.ewald_corrections:
        flags |= _lib.DYN_FLAG_EWALD_CORRECTIONS
    if cfg.full_energy:
        flags |= _lib.DYN_FLAG_FULL_ENERGY
    if cfg.zero_com_drift:
        flags |= _lib.DYN_FLAG_COM_REMOVAL
    if cfg.recenter_sim_box:
        flags |= _lib.DYN_FLAG_RECENTER
    if cfg.reset_angle:
        flags |= _lib.DYN_FLAG_RESET_ANGLE
    if cfg.rattle_velocities:
        flags |= _lib.DYN_FLAG_RATTLE_VELOCITIES
    c.flags = flags
    if cfg.alch_range is not None:
        c.alch_begin, c.alch_end = int(cfg.alch_range[0]), int(cfg.alch_range[1])
    c.alch_lambda = float(cfg.alch_lambda)
    c.thermo_dof = thermo_dof(system, cfg)
    c.seed = int(cfg.seed) & 0xFFFFFFFFFFFFFFFF
    c.ww_union_chunk = int(cfg.ww_union_chunk)
    c.prune_buffer = float(cfg.prune_buffer)
    c.spme_brick_cap = int(cfg.spme_brick_cap)
    c.pair_item_entries = int(cfg.pair_item_entries)
    c.ww_split = int(cfg.ww_split)
    c.lincs_order = int(cfg.lincs_order)
    c.lincs_iter = int(cfg.lincs_iter)
    return c


def _system_desc(system):
    """dyn_system_desc_t for a system dict; returns (desc, arrays kept alive,
    n_water, n_atoms)."""
    wp = f32(system.get("water_pos", np.zeros((0, 3, 3)))).reshape(-1, 9)
    wv = f32(system.get("water_vel", np.zeros_like(wp))).reshape(-1, 9)
    ap = f32(system.get("atom_pos", np.zeros((0, 3)))).reshape(-1, 3)
    na = len(ap)
    nw = len(wp)
    keep = {}

    def arr(name, conv, shape=None):
        if name not in system or system[name] is None or len(system[name]) == 0:
            return None
        a = conv(system[name])
        if shape is not None:
            a = a.reshape(shape)
        keep[name] = a
        return a

    d = _lib.SystemDesc()
    d.n_atoms = na
    d.atom_pos = ptr(arr("atom_pos", f32, -1))
    d.atom_vel = ptr(arr("atom_vel", f32, -1))
    d.atom_mass = ptr(arr("atom_mass", f32))
    d.atom_q = ptr(arr("atom_q", f32))
    d.atom_sigma = ptr(arr("atom_sigma", f32))
    d.atom_eps = ptr(arr("atom_eps", f32))
    d.atom_static = ptr(arr("atom_static", u8))
    d.n_water = nw
    keep["wp"] = np.ascontiguousarray(wp)
    keep["wv"] = np.ascontiguousarray(wv)
    d.water_pos = ptr(keep["wp"]) if nw else None
    d.water_vel = ptr(keep["wv"]) if nw else None
    for name in ("excl", "pair14"):
        a = arr(name, u32, -1)
        setattr(d, "n_" + name, 0 if a is None else len(a) // 2)
        setattr(d, name, ptr(a))
    b = arr("bonds", u32, -1)
    d.n_bonds = 0 if b is None else len(b) // 2
    d.bonds = ptr(b)
    d.bond_k = ptr(arr("bond_k", f32))
    d.bond_r0 = ptr(arr("bond_r0", f32))
    a = arr("angles", u32, -1)
    d.n_angles = 0 if a is None else len(a) // 3
    d.angles = ptr(a)
    d.angle_k = ptr(arr("angle_k", f32))
    d.angle_theta0 = ptr(arr("angle_theta0", f32))
    dh = arr("dihedrals", u32, -1)
    d.n_dihedrals = 0 if dh is None else len(dh) // 4
    d.dihedrals = ptr(dh)
    d.dihedral_k = ptr(arr("dihedral_k", f32))
    d.dihedral_n = ptr(arr("dihedral_n", f32))
    d.dihedral_phase = ptr(arr("dihedral_phase", f32))
    cn = arr("constraints", u32, -1)
    d.n_constraints = 0 if cn is None else len(cn) // 2
    d.constraints = ptr(cn)
    d.constraint_r0 = ptr(arr("constraint_r0", f32))
    return d, keep, nw, na


class MdState:
    """A device-resident simulation (MdState, src/lib.rs:610-705)."""

    def __init__(self, system, cfg=None, stream=None):
        self.cfg = cfg or MdConfig()
        self.system = system
        d, keep, self.n_water, self.n_atoms = _system_desc(system)
        c = _config_struct(system, self.cfg)
        h = C.c_void_p()
        check(lib().dyn_sys_create(stream, C.byref(c), C.byref(d), C.byref(h)))
        self._h = h
        self._owned = True
        self._cstruct = c
        self._static = np.asarray(system.get("atom_static", np.zeros(self.n_atoms, bool)), bool).reshape(-1)
        self._snapshots = []
        if self.cfg.snapshot_memory:
            self.enable_snapshots(self.cfg.snapshot_memory, self.cfg.snapshot_capacity, velocities=True)

    @classmethod
    def _member(cls, handle, system, cfg):
        """A view of a batch member (owned by the batch, never destroyed here)."""
        self = cls.__new__(cls)
        self.cfg = cfg
        self.system = system
        self.n_water = len(np.asarray(system.get("water_pos", np.zeros((0, 3, 3)))).reshape(-1, 9))
        self.n_atoms = len(np.asarray(system.get("atom_pos", np.zeros((0, 3)))).reshape(-1, 3))
        self._h = handle
        self._owned = False
        self._static = np.asarray(system.get("atom_static", np.zeros(self.n_atoms, bool)), bool).reshape(-1)
        return self

    @property
    def handle(self):
        if self._h is None:
            raise _lib.DynError(_lib.DYN_ERR_INVALID, "MdState already closed")
        return self._h

    def step(self, dt, n_steps=1):
        """Advance n_steps of dt ps (asynchronous; see sync())."""
        check(lib().dyn_sys_step(self.handle, int(n_steps), float(dt)))

    def sync(self):
        check(lib().dyn_sys_sync(self.handle))

    def energies(self):
        e = _lib.Energies()
        check(lib().dyn_sys_get_energies(self.handle, C.byref(e)))
        return e.as_dict()

    def forces(self):
        """One force evaluation (reset_f_acc_pe_virial + apply_all_forces,
        src/lib.rs:1220-1348): dict with f_atoms (n,3), f_water (nw,4,3)
        sites O, H0, H1, M, and the energies."""
        fa = np.zeros((max(self.n_atoms, 1), 3))
        fw = np.zeros((max(self.n_water, 1), 4, 3))
        e = _lib.Energies()
        check(lib().dyn_sys_forces(self.handle, ptr(fa), ptr(fw), C.byref(e)))
        out = e.as_dict()
        out["f_atoms"] = fa[:self.n_atoms]
        out["f_water"] = fw[:self.n_water]
        return out

    def state(self):
        na, nw = self.n_atoms, self.n_water
        ap = np.zeros((max(na, 1), 3), np.float32)
        av = np.zeros((max(na, 1), 3), np.float32)
        wp = np.zeros((max(nw, 1), 3, 3), np.float32)
        wv = np.zeros((max(nw, 1), 3, 3), np.float32)
        wm = np.zeros((max(nw, 1), 3), np.float32)
        check(lib().dyn_sys_get_state(self.handle, ptr(ap), ptr(av), ptr(wp), ptr(wv), ptr(wm)))
        return {"atom_pos": ap[:na], "atom_vel": av[:na], "water_pos": wp[:nw],
                "water_vel": wv[:nw], "water_m": wm[:nw]}

    def step_host(self, dt, n_steps, inputs, outputs):
        """dyn_sys_step_host: host buffers in, n steps, host buffers out.

        ``inputs`` / ``outputs``: dicts with optional atom_pos, atom_vel,
        water_pos, water_vel float32 arrays (home order; page-locked for full
        bandwidth).  Returns the energies dict."""
        keys = ("atom_pos", "atom_vel", "water_pos", "water_vel")
        e = _lib.Energies()
        check(lib().dyn_sys_step_host(self.handle, int(n_steps), float(dt),
                                      *[ptr(inputs.get(k)) for k in keys],
                                      *[ptr(outputs.get(k)) for k in keys], C.byref(e)))
        return e.as_dict()

    STAGES = ("first_half", "list", "pairs", "bonded", "spme", "kick_finalize",
              "pairs_water_water", "pairs_water_atom", "pairs_atom_atom",
              "spme_spread", "spme_fft_convolve", "spme_gather", "spme_corrections")

    def stage_times(self, dt, n_steps):
        """Mean ms per step of each stage, timed with CUDA events."""
        ms = np.zeros(_lib.DYN_STAGES)
        check(lib().dyn_sys_stage_times(self.handle, int(n_steps), float(dt), ptr(ms)))
        return dict(zip(self.STAGES, ms.tolist()))

    def memory(self):
        """Device bytes this system holds."""
        b = C.c_uint64()
        check(lib().dyn_sys_memory(self.handle, C.byref(b)))
        return b.value

    def set_lambda(self, lam):
        """Another lambda window for the alchemical molecule; forces are
        evaluated again at once."""
        check(lib().dyn_sys_set_lambda(self.handle, float(lam)))
        self.cfg.alch_lambda = float(lam)

    def set_static(self, mask=None):
        """Atoms held fixed (bool (n_atoms,), None = none), with the
        thermostat's degrees of freedom following (dof_for_thermo)."""
        na = self.n_atoms
        m = np.zeros(na, bool) if mask is None else np.asarray(mask, bool).reshape(na)
        sysd = dict(self.system, atom_static=m)
        mu = np.ascontiguousarray(m, np.uint8)  # alive through the call
        check(lib().dyn_sys_set_static(self.handle, ptr(mu) if na else None, int(thermo_dof(sysd, self.cfg))))
        self._static = m

    def relax_solvent(self, n_steps=200, dt=0.0005):
        """The solvent relaxes around the frozen solute: every atom static
        for ``n_steps`` steps of ``dt`` ps, then the atoms' own static
        flags back (MdState::md_on_solute_only, src/solvent/init.rs:773-805;
        200 steps of 0.5 fs are the reference's values for water,
        :64-69)."""
        keep = self._static.copy()
        self.set_static(np.ones(self.n_atoms, bool))
        try:
            self.step(dt, n_steps)
        finally:
            self.set_static(keep)

    def minimize_energy(self, max_iters=1000, tolerance=1000.0 * 0.0239005):
        """Steepest-descent relaxation of the atoms on the device
        (MdState::minimize_energy, src/minimize_energy.rs:60-260; the
        defaults are the reference's max_init_relaxation_iters and
        energy_minimization_tolerance, src/config.rs:122-126).  Returns
        (accepted steps, potential energy of the atom terms without the
        reciprocal part, kcal/mol)."""
        it, e = C.c_uint32(), C.c_double()
        check(lib().dyn_sys_minimize(self.handle, int(max_iters), float(tolerance), C.byref(it), C.byref(e)))
        return it.value, e.value

    def enable_snapshots(self, ratio, capacity=256, velocities=False, forces=False):
        """Record a snapshot into a device ring every ``ratio`` steps
        (SnapshotHandlers.memory, src/snapshot.rs:33-57 and 753-776): the
        step graph writes the frames; read_snapshots() copies them out.
        ratio 0 stops recording."""
        fields = (_lib.DYN_SNAP_VELOCITIES if velocities else 0) | (_lib.DYN_SNAP_FORCES if forces else 0)
        check(lib().dyn_sys_snapshots(self.handle, int(ratio), int(capacity), fields))
        self._snap = (int(ratio), int(capacity), bool(velocities), bool(forces))

    def read_snapshots(self, max_frames=None):
        """The frames recorded since the last read, oldest first: a list of
        dicts with step, time_ps, energies, box, ``pos`` (n_sites, 3) in the
        layout atoms (wrapped into the box) then O, H0, H1 of each water,
        ``vel`` (same layout) and ``force`` (n_atoms, 3) when recorded, and
        ``lost`` on the first frame (frames overwritten unread)."""
        ratio, cap, with_v, with_f = getattr(self, "_snap", (0, 0, False, False))
        if not ratio:
            return []
        n = cap if max_frames is None else min(cap, int(max_frames))
        ns = self.n_atoms + 3 * self.n_water
        pos = np.zeros((n, ns, 3), np.float32)
        vel = np.zeros((n, ns, 3), np.float32) if with_v else None
        frc = np.zeros((n, max(self.n_atoms, 1), 3), np.float32) if with_f else None
        frames = (_lib.Frame * max(n, 1))()
        got, lost = C.c_uint32(), C.c_uint64()
        check(lib().dyn_sys_snapshots_read(self.handle, n, ptr(pos), ptr(vel) if with_v else None,
                                           ptr(frc) if with_f and self.n_atoms else None, C.addressof(frames),
                                           C.byref(got), C.byref(lost)))
        out = []
        for i in range(got.value):
            d = frames[i].as_dict()
            d["pos"] = pos[i]
            if with_v:
                d["vel"] = vel[i]
            if with_f:
                d["force"] = frc[i][:self.n_atoms]
            out.append(d)
        if out:
            out[0]["lost"] = lost.value
        return out

    @property
    def snapshots(self):
        """The snapshots recorded so far (MdState.snapshots,
        src/lib.rs:635-637), oldest first, as Snapshot objects; frames still
        in the device ring are copied out first."""
        na, nw = self.n_atoms, self.n_water
        for d in self.read_snapshots():
            pos = d["pos"]
            w = pos[na:].reshape(nw, 3, 3)
            vel = d.get("vel")
            e = SnapshotEnergyData(
                energy_kinetic=d["kinetic"], energy_potential=d["potential"],
                energy_potential_nonbonded=d["potential"] - d["potential_bonded"],
                energy_potential_bonded=d["potential_bonded"], temperature=d["temperature"],
                pressure=d["pressure_bar"], dh_dl=d["dh_dl"] if self.cfg.alch_range else None,
                volume=d["volume"], density=d["density"])
            self._snapshots.append(Snapshot(
                time=d["time_ps"], step=d["step"], atom_posits=pos[:na], water_o_posits=w[:, 0],
                water_h0_posits=w[:, 1], water_h1_posits=w[:, 2], energy_data=e,
                cell=(tuple(d["box_lo"]), tuple(d["box_hi"])),
                atom_velocities=None if vel is None else vel[:na],
                water_velocities=None if vel is None else vel[na:].reshape(nw, 3, 3)[:, 0],
                force=d.get("force")))
        return self._snapshots

    def __str__(self):
        e = self.energies()
        return (f"MdState: {self.n_atoms} atoms, {self.n_water} waters, step {e['step']}, "
                f"T {e['temperature']:.2f} K, PE {e['potential']:.3f} kcal/mol")

    def launches_per_step(self, spme=True):
        """Kernels of a step without a list rebuild or periodic task."""
        n = C.c_uint32()
        check(lib().dyn_sys_launches_per_step(self.handle, 1 if spme else 0, C.byref(n)))
        return n.value

    def launches_conditional(self):
        """(kernels added by a list rebuild, kernels added by a periodic task)."""
        r, p = C.c_uint32(), C.c_uint32()
        check(lib().dyn_sys_launches_conditional(self.handle, C.byref(r), C.byref(p)))
        return r.value, p.value

    def list_pairs(self, kind):
        """The pairs the pair kernels evaluate now (dyn_sys_list_pairs):
        kind 0 water-water (water, water), 1 water-atom (water, atom),
        2 atom-atom; an (n, 2) uint32 array of original indices."""
        n = C.c_uint64(0)
        check(lib().dyn_sys_list_pairs(self.handle, int(kind), None, 0, C.byref(n)))
        out = np.zeros((max(int(n.value), 1), 2), np.uint32)
        check(lib().dyn_sys_list_pairs(self.handle, int(kind), ptr(out), int(n.value), C.byref(n)))
        return out[:int(n.value)]

    def set_state(self, atom_pos=None, atom_vel=None, water_pos=None, water_vel=None):
        conv = [None if x is None else f32(x).reshape(-1) for x in (atom_pos, atom_vel, water_pos, water_vel)]
        check(lib().dyn_sys_set_state(self.handle, *[ptr(x) for x in conv]))

    def close(self):
        if self._h is not None:
            if self._owned:
                lib().dyn_sys_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MdBatch:
    """Independent systems advanced together (dyn_batch_*): every stage of a
    step is one kernel launch over all members with per-member block ranges,
    and a step is one CUDA graph.  ``members[i]`` is an MdState view of
    system i (state, energies, forces); results equal running it alone.
    With ``tune``, each member takes the autotuner's choice for its size
    class (dynamics_b200.tune; classes not yet in the cache are tuned
    first, one representative member each)."""

    def __init__(self, systems=(), cfgs=(), stream=None, tune=False):
        systems = list(systems)
        if isinstance(cfgs, MdConfig):
            cfgs = [cfgs] * len(systems)
        cfgs = list(cfgs)
        if tune:
            from . import tune as _tune
            import dataclasses as _dc
            # the tuner times systems alone; in a batch the members keep their
            # own ww_split (0: none, as the batch fills the GPU)
            cfgs = [_dc.replace(_tune.apply_tuned(s, c, tune_missing=True, stream=stream), ww_split=c.ww_split)
                    for s, c in zip(systems, cfgs)]
        self.cfgs = cfgs
        n = len(systems)
        descs = (_lib.SystemDesc * max(n, 1))()
        confs = (_lib.Config * max(n, 1))()
        keep = []
        for i, (sysd, cfg) in enumerate(zip(systems, cfgs)):
            d, k, _, _ = _system_desc(sysd)
            descs[i] = d
            confs[i] = _config_struct(sysd, cfg)
            keep.append(k)
        h = C.c_void_p()
        check(lib().dyn_batch_create(stream, n, confs, descs, C.byref(h)))
        self._h = h
        self.members = []
        for i in range(n):
            m = C.c_void_p()
            check(lib().dyn_batch_member(h, i, C.byref(m)))
            self.members.append(MdState._member(m, systems[i], cfgs[i]))

    def step(self, dt, n_steps=1):
        check(lib().dyn_batch_step(self._h, int(n_steps), float(dt)))

    def sync(self):
        check(lib().dyn_batch_sync(self._h))

    def add(self, system, cfg):
        """Adds a member between steps (continuous batching); returns its
        MdState view."""
        d, keep, _, _ = _system_desc(system)
        c = _config_struct(system, cfg)
        idx = C.c_uint32()
        check(lib().dyn_batch_add(self._h, C.byref(c), C.byref(d), C.byref(idx)))
        h = C.c_void_p()
        check(lib().dyn_batch_member(self._h, idx.value, C.byref(h)))
        m = MdState._member(h, system, cfg)
        self.members.append(m)
        return m

    def remove(self, member):
        """Removes (destroys) a member between steps."""
        i = self.members.index(member)
        check(lib().dyn_batch_remove(self._h, i))
        member._h = None
        del self.members[i]

    def memory(self):
        b = C.c_uint64()
        check(lib().dyn_batch_memory(self._h, C.byref(b)))
        return b.value

    def state_layout(self):
        """Member offsets (floats) into the packed host state, n + 1 entries."""
        off = np.zeros(len(self.members) + 1, np.uint64)
        check(lib().dyn_batch_state_layout(self._h, ptr(off)))
        return off

    def host_buffer(self):
        """The batch's page-locked packed-state area as a float32 array (valid
        until the batch grows or closes)."""
        buf, n = C.POINTER(C.c_float)(), C.c_uint64()
        check(lib().dyn_batch_host_buffer(self._h, C.byref(buf), C.byref(n)))
        return np.ctypeslib.as_array(buf, shape=(max(n.value, 1),))[:n.value]

    def unpack(self, packed, i):
        """Views of member i's atom_pos, atom_vel, water_pos, water_vel in a
        packed state array."""
        off = self.state_layout()
        m = self.members[i]
        na, nw = m.n_atoms, m.n_water
        a = packed[int(off[i]):int(off[i + 1])]
        return {"atom_pos": a[:3 * na].reshape(na, 3), "atom_vel": a[3 * na:6 * na].reshape(na, 3),
                "water_pos": a[6 * na:6 * na + 9 * nw].reshape(nw, 3, 3),
                "water_vel": a[6 * na + 9 * nw:].reshape(nw, 3, 3)}

    def step_host(self, dt, n_steps=1, state_in=None, state_out=None, energies=False):
        """dyn_batch_step_host: every member's packed state in (state_in,
        None keeps the resident states), n steps, packed state out
        (state_out, None skips it); one copy each way for the whole batch.
        Returns the members' energies dicts with energies, else None."""
        n = len(self.members)
        total = int(self.state_layout()[-1])
        for a in (state_in, state_out):
            if a is not None and (a.dtype != np.float32 or a.size < total or not a.flags["C_CONTIGUOUS"]):
                raise ValueError(f"packed state: contiguous float32 with at least {total} values")
        e = (_lib.Energies * max(n, 1))() if energies else None
        check(lib().dyn_batch_step_host(self._h, int(n_steps), float(dt), ptr(state_in), ptr(state_out),
                                        e if energies else None))
        return [e[i].as_dict() for i in range(n)] if energies else None

    def launches(self, spme=True):
        """(fixed, rebuild, periodic) batched launches of one step."""
        f, r, p = C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(lib().dyn_batch_launches(self._h, 1 if spme else 0, C.byref(f), C.byref(r), C.byref(p)))
        return f.value, r.value, p.value

    def close(self):
        if self._h is not None:
            for m in self.members:
                m._h = None
            lib().dyn_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def equilibrate(system, cfg, n_steps=1000, dt=0.001, gamma=50.0):
    """Relax a freshly generated system with strongly damped Langevin
    dynamics on the device and return a copy with the new positions and
    velocities.  Plays the role of the reference's start-up relaxation
    (minimize_energy and the solvent-only MD of MdState::new,
    src/lib.rs:1106-1112) for synthetic inputs."""
    import copy
    c = copy.deepcopy(cfg)
    c.integrator = LangevinMiddle(gamma=gamma)
    c.spme_interval = 1
    c.energy_interval = max(1, n_steps)
    st = MdState(system, c)
    st.step(dt, n_steps)
    s = st.state()
    st.close()
    out = dict(system)
    out["water_pos"] = s["water_pos"]
    out["water_vel"] = s["water_vel"]
    if len(s["atom_pos"]):
        out["atom_pos"] = s["atom_pos"]
        out["atom_vel"] = s["atom_vel"]
    return out
