"""The stochastic and pressure half of the step vs the float64 oracle.

The engine draws its noise from Philox4x32-10 keyed by (particle, step,
seed); oracle.philox reproduces that stream bit for bit, so stochastic steps
can be compared step for step:

* Langevin-middle (src/integrate.rs:100-212; the OU step of
  apply_langevin_thermostat, src/thermostat.rs:308-362);
* velocity Verlet with the CSVR thermostat (src/integrate.rs:213-317,
  src/thermostat.rs:258-304), on the rigid-body kinetic energy;
* the C-rescale barostat (src/barostat.rs:329-413, which the reference
  leaves disabled at :367-368), driven by the molecular pressure.

Waters plus chain molecules (exclusions, 1-4 pairs, bonded terms), SPME
every step, no COM removal or recentering.  Tolerances: positions within
1e-4 A and velocities within 1e-4 relative RMS of the oracle after the
steps (the float32 engine against float64), as for the deterministic
velocity-Verlet trajectory; temperature and pressure within 1e-5 relative
of the oracle's (of the pressure's kinetic and virial terms).
"""
import numpy as np
import pytest

from dynamics_b200 import md, synth
from oracle import integrate as oint
from oracle import method

from .systems import mixed, rel_rms

pytestmark = pytest.mark.gpu

POS_ATOL = 1e-4
VEL_RTOL = 1e-4
SCALAR_RTOL = 1e-5
CUTOFF = 8.0


def _cfg(sysd, integ, **kw):
    ext = sysd["box_hi"] - sysd["box_lo"]
    grid = tuple(int(2 ** np.ceil(np.log2(x))) for x in ext)
    return md.MdConfig(coulomb_cutoff=CUTOFF, lj_cutoff=CUTOFF, spme_alpha=synth.ewald_alpha(CUTOFF),
                       spme_grid=grid, integrator=integ, spme_interval=1, zero_com_drift=False,
                       recenter_sim_box=False, reset_angle=False, **kw)


class _Oracle:
    """float64 state of the system and its force function; the box is
    mutable (the barostat scales it)."""

    def __init__(self, sysd, cfg):
        self.sysd, self.cfg = sysd, cfg
        self.lo = sysd["box_lo"].astype(np.float64)
        self.ext = (sysd["box_hi"] - sysd["box_lo"]).astype(np.float64)
        na = len(sysd["atom_pos"])
        self.s = {
            "atom_pos": sysd["atom_pos"].astype(np.float64), "atom_vel": sysd["atom_vel"].astype(np.float64),
            "atom_mass": sysd["atom_mass"].astype(np.float64), "atom_static": np.zeros(na, bool),
            "water_pos": sysd["water_pos"].astype(np.float64), "water_vel": sysd["water_vel"].astype(np.float64),
        }
        f = self.forces(self.s)
        oint.kick_and_calc_accel(self.s, f, 0.0)

    def forces(self, s):
        d = dict(self.sysd)
        d["atom_pos"], d["water_pos"] = s["atom_pos"], s["water_pos"]
        d["box_lo"] = self.lo.astype(np.float32)
        d["box_hi"] = (self.lo + self.ext).astype(np.float32)
        d.pop("water_m", None)
        f = method.all_forces(d, {"cutoff": CUTOFF, "lj_cutoff": CUTOFF,
                                  "alpha": float(np.float32(self.cfg.spme_alpha)),
                                  "grid": self.cfg.spme_grid, "mode": "reference"})
        s["water_m"] = method.water_sites(d)[:, 3]
        return f


def _compare_state(got, s, ext):
    d = got["water_pos"].astype(np.float64) - s["water_pos"]
    d -= np.round(d / ext) * ext
    da = got["atom_pos"].astype(np.float64) - s["atom_pos"]
    da -= np.round(da / ext) * ext
    pos_err = max(float(np.max(np.abs(d))), float(np.max(np.abs(da))))
    vel_err = rel_rms(np.concatenate([got["water_vel"].reshape(-1), got["atom_vel"].reshape(-1)]),
                      np.concatenate([s["water_vel"].reshape(-1), s["atom_vel"].reshape(-1)]))
    return pos_err, vel_err


def test_langevin_middle_matches_oracle(gpu_lib):
    sysd = mixed()
    gamma, seed, dt, n = 5.0, 11, 0.002, 5
    cfg = _cfg(sysd, md.LangevinMiddle(gamma=gamma), seed=seed)
    st = md.MdState(sysd, cfg)
    st.step(dt, n)
    got = st.state()
    st.close()
    o = _Oracle(sysd, cfg)
    for k in range(n):
        oint.step_langevin_middle(o.s, o.forces, dt, gamma, cfg.temp_target, k, seed, o.lo, o.ext)
    pos_err, vel_err = _compare_state(got, o.s, o.ext)
    assert pos_err < POS_ATOL, pos_err
    assert vel_err < VEL_RTOL, vel_err
    # the noise is not negligible next to the tolerance: without it the
    # velocities differ from the stochastic run's by far more
    q = _Oracle(sysd, cfg)
    for k in range(n):
        oint.step_langevin_middle(q.s, q.forces, dt, 0.0, cfg.temp_target, k, seed, q.lo, q.ext)
    assert _compare_state(got, q.s, q.ext)[1] > 100 * VEL_RTOL


def test_csvr_matches_oracle(gpu_lib):
    sysd = mixed()
    tau, seed, dt, n = 0.1, 5, 0.002, 5
    cfg = _cfg(sysd, md.VerletVelocity(thermostat=tau), seed=seed)
    dof = md.thermo_dof(sysd, cfg)
    st = md.MdState(sysd, cfg)
    temps = []
    for _ in range(n):
        st.step(dt, 1)
        temps.append(st.energies()["temperature"])
    got = st.state()
    st.close()
    o = _Oracle(sysd, cfg)
    lams = []
    for k in range(n):
        _, lam, _, _, o.lo, o.ext = oint.step_verlet_csvr(o.s, o.forces, dt, tau, cfg.temp_target, dof, k, seed,
                                                          o.lo, o.ext)
        lams.append(lam)
        t_ref = 2.0 * oint.rigid_kinetic_energy(o.s, o.ext) / (dof * oint.opc.GAS_CONST_R)
        assert abs(temps[k] - t_ref) <= SCALAR_RTOL * t_ref, (k, temps[k], t_ref)
    pos_err, vel_err = _compare_state(got, o.s, o.ext)
    assert pos_err < POS_ATOL, pos_err
    assert vel_err < VEL_RTOL, vel_err
    # the thermostat acted: its scale factors are far from 1 next to the tolerance
    assert max(abs(x - 1.0) for x in lams) > 20 * VEL_RTOL, lams


def test_crescale_matches_oracle(gpu_lib):
    """Two steps of velocity Verlet + CSVR + C-rescale.  A larger
    compressibility and shorter coupling time than the defaults make the
    box change (~1e-3 per step) large enough to compare in float32."""
    sysd = mixed()
    tau, seed, dt, n = 0.1, 9, 0.002, 2
    baro = {"p_target": 1.0, "tau": 0.5, "kappa": 4.5e-4}
    cfg = _cfg(sysd, md.VerletVelocity(thermostat=tau), seed=seed,
               barostat_cfg=md.BarostatCfg(pressure_target=baro["p_target"], tau=baro["tau"],
                                           solvent_compressibility=baro["kappa"]))
    dof = md.thermo_dof(sysd, cfg)
    st = md.MdState(sysd, cfg)
    en = []
    for _ in range(n):
        st.step(dt, 1)
        en.append(st.energies())
    got = st.state()
    st.close()
    o = _Oracle(sysd, cfg)
    ext0 = o.ext.copy()
    for k in range(n):
        f, lam, mu, p, o.lo, o.ext = oint.step_verlet_csvr(o.s, o.forces, dt, tau, cfg.temp_target, dof, k, seed,
                                                           o.lo, o.ext, baro=baro)
        # the pressure's scale: its kinetic and virial terms
        vol = float(np.prod(o.ext / mu))
        scale = (2.0 * oint.kinetic_energy_translational(o.s) + abs(f["virial"])) / (3.0 * vol) * \
            oint.opc.BAR_PER_KCAL_MOL_PER_ANSTROM_CUBED
        assert abs(en[k]["pressure_bar"] - p) <= SCALAR_RTOL * scale, (k, en[k]["pressure_bar"], p, scale)
        np.testing.assert_allclose(np.asarray(en[k]["box"], np.float64), o.ext, rtol=1e-6)
    assert np.max(np.abs(o.ext / ext0 - 1.0)) > 1e-4, "the box did not change measurably"
    pos_err, vel_err = _compare_state(got, o.s, o.ext)
    assert pos_err < POS_ATOL, pos_err
    assert vel_err < VEL_RTOL, vel_err


@pytest.mark.parametrize("mode", ["reference", "corrected"])
def test_virial_components_match_oracle(gpu_lib, mode):
    """The parts of the virial that feed the pressure vs the float64 oracle:
    short-range pairs (1-4 pairs included), reciprocal space with the 1-4
    vacuum correction (reference mode, src/non_bonded.rs:763-790) or the
    Ewald exclusion corrections (corrected mode), and the bonded terms.
    Each within 1e-5 of the sum of their magnitudes."""
    sysd = mixed()
    cfg = _cfg(sysd, md.VerletVelocity(thermostat=None), ewald_corrections=(mode == "corrected"),
               full_energy=(mode == "corrected"))
    st = md.MdState(sysd, cfg)
    got = st.forces()
    m = st.state()["water_m"]
    st.close()
    ref = method.all_forces({**sysd, "water_m": m}, {
        "cutoff": CUTOFF, "lj_cutoff": CUTOFF, "alpha": float(np.float32(cfg.spme_alpha)),
        "grid": cfg.spme_grid, "mode": mode})
    pairs = [("virial_short", ref["virial_short"]),
             ("virial_recip", ref["virial_recip"] + ref["virial_corr"]),
             ("virial_bonded", ref["virial_bonded"])]
    scale = sum(abs(r) for _, r in pairs)
    errs = {k: (got[k], r, abs(got[k] - r) / scale) for k, r in pairs}
    print(mode, errs)
    for k, (g, r, e) in errs.items():
        assert e <= SCALAR_RTOL, (k, g, r, e)
