"""ff19SB peptides in OPC water with ions and bond-to-H constraints: forces
against the float64 oracle, a constrained velocity-Verlet trajectory against
the oracle's restatement of lincs_hydrogens / rattle_hydrogens
(src/bonded.rs:218-304), and constraint satisfaction under Langevin
dynamics."""
import numpy as np
import pytest

from dynamics_b200 import md, peptide, synth
from oracle import integrate as oint

from .systems import rel_rms
from .test_gpu_native import FORCE_RTOL, PE_RTOL, _cfg, _compare, _oracle

pytestmark = pytest.mark.gpu


def _system(seed=4):
    sysd, _ = peptide.solvated_system(28.0, 700, n_res=(10,), seed=seed, nacl_molar=0.15)
    return sysd


@pytest.fixture(scope="module")
def relaxed():
    sysd = _system()
    return md.equilibrate(sysd, _cfg(sysd), n_steps=200, dt=0.0005)


@pytest.mark.parametrize("mode", ["reference", "corrected"])
def test_peptide_forces_match_oracle(gpu_lib, relaxed, mode):
    cfg = _cfg(relaxed, mode)
    st = md.MdState(relaxed, cfg)
    got = st.forces()
    ref = _oracle(relaxed, cfg, st)
    err = _compare(got, ref)
    assert err < FORCE_RTOL, f"force rel-RMS {err:.3e}"
    assert abs(got["potential"] - ref["pe"]) <= PE_RTOL * abs(ref["pe"]), (got["potential"], ref["pe"])
    st.close()


@pytest.mark.parametrize("rattle_velocities", [False, True])
def test_constrained_trajectory_matches_oracle(gpu_lib, relaxed, rattle_velocities):
    cfg = _cfg(relaxed, integ=md.VerletVelocity(thermostat=None), spme_interval=1, zero_com_drift=False,
               recenter_sim_box=False, reset_angle=False, rattle_velocities=rattle_velocities)
    st = md.MdState(relaxed, cfg)
    n, dt = 5, 0.002
    st.step(dt, n)
    got = st.state()
    s = {"atom_pos": relaxed["atom_pos"].astype(np.float64), "atom_vel": relaxed["atom_vel"].astype(np.float64),
         "atom_mass": relaxed["atom_mass"].astype(np.float64),
         "atom_static": np.zeros(len(relaxed["atom_pos"]), bool),
         "water_pos": relaxed["water_pos"].astype(np.float64),
         "water_vel": relaxed["water_vel"].astype(np.float64),
         "constraints": relaxed["constraints"], "constraint_r0": relaxed["constraint_r0"]}
    lo = relaxed["box_lo"].astype(np.float64)
    ext = (relaxed["box_hi"] - relaxed["box_lo"]).astype(np.float64)

    def forces(s):
        d = dict(relaxed)
        d["atom_pos"], d["water_pos"] = s["atom_pos"], s["water_pos"]
        d.pop("water_m", None)
        return _oracle(d, cfg)

    oint.kick_and_calc_accel(s, forces(s), 0.0)
    for _ in range(n):
        oint.kick_and_drift(s, dt / 2, dt, lo, ext, rattle_velocities=rattle_velocities)
        oint.kick_and_calc_accel(s, forces(s), dt / 2)
    d = got["atom_pos"].astype(np.float64) - s["atom_pos"]
    d -= np.round(d / ext) * ext
    assert np.max(np.abs(d)) < 2e-4
    assert rel_rms(got["atom_vel"], s["atom_vel"]) < 2e-3
    st.close()


def test_constraints_hold_under_langevin(gpu_lib, relaxed):
    cfg = _cfg(relaxed, integ=md.LangevinMiddle(gamma=1.0))
    st = md.MdState(relaxed, cfg)
    st.step(0.002, 100)
    e = st.energies()
    assert np.isfinite(e["temperature"]) and 150.0 < e["temperature"] < 600.0
    p = st.state()["atom_pos"].astype(np.float64)
    c = relaxed["constraints"].astype(int)
    r = np.linalg.norm(p[c[:, 0]] - p[c[:, 1]], axis=1)
    assert np.max(np.abs(r - relaxed["constraint_r0"]) / relaxed["constraint_r0"]) < 1e-3
    st.close()


def test_rattle_velocities_conserve_energy(gpu_lib, relaxed):
    """Velocity Verlet without thermostat: with the velocities following
    the constraint corrections the total energy holds; the reference's
    position-only correction loses kinetic energy every step."""
    drift = {}
    for rv in (False, True):
        cfg = _cfg(relaxed, "corrected", integ=md.VerletVelocity(thermostat=None), spme_interval=1,
                   zero_com_drift=False, recenter_sim_box=False, reset_angle=False, rattle_velocities=rv)
        st = md.MdState(relaxed, cfg)
        e = []
        for _ in range(20):
            st.step(0.002, 25)
            en = st.energies()
            e.append(en["kinetic_rigid"] + en["potential"])
        st.close()
        drift[rv] = np.polyfit(np.arange(len(e)), np.array(e), 1)[0]
    assert abs(drift[True]) < 0.25 * abs(drift[False]), drift


def test_minimizer_matches_oracle(gpu_lib):
    """Steepest descent on the device against the float64 restatement of
    src/minimize_energy.rs: same accepted steps, positions and energy."""
    from oracle import minimize as omin
    sysd = _system(seed=9)
    cfg = _cfg(sysd)
    st = md.MdState(sysd, cfg)
    n_it, e = st.minimize_energy(max_iters=12, tolerance=0.0)
    got = st.state()["atom_pos"].astype(np.float64)
    st.close()
    params = {"cutoff": cfg.coulomb_cutoff, "lj_cutoff": cfg.lj_cutoff,
              "alpha": float(np.float32(cfg.spme_alpha)), "grid": cfg.spme_grid, "mode": "reference"}
    x, n_ref, e_ref = omin.minimize_energy(sysd, params, 12, 0.0)
    assert n_it == n_ref == 12
    assert abs(e - e_ref) <= 1e-5 * abs(e_ref), (e, e_ref)
    box = (sysd["box_hi"] - sysd["box_lo"]).astype(np.float64)
    d = got - x
    d -= np.round(d / box) * box
    assert np.max(np.abs(d)) < 2e-3


def test_minimizer_lowers_energy_and_forces(gpu_lib):
    sysd = _system(seed=10)
    cfg = _cfg(sysd)
    st = md.MdState(sysd, cfg)
    f0 = np.linalg.norm(st.forces()["f_atoms"], axis=1).max()
    n_it, e = st.minimize_energy(max_iters=300)
    f1 = np.linalg.norm(st.forces()["f_atoms"], axis=1).max()
    assert 0 < n_it <= 300 and np.isfinite(e)
    assert f1 < f0
    st.step(0.002, 20)  # the system runs on from the minimized geometry
    assert np.isfinite(st.energies()["temperature"])
    st.close()


def test_relax_solvent_holds_the_solute(gpu_lib):
    """md_on_solute_only: the atoms stay put while the waters move; the
    atoms' own static flags come back afterwards."""
    sysd = _system(seed=11)
    cfg = _cfg(sysd, integ=md.LangevinMiddle(gamma=1.0))
    st = md.MdState(sysd, cfg)
    a0 = st.state()
    st.relax_solvent(n_steps=50, dt=0.0005)
    a1 = st.state()
    np.testing.assert_array_equal(a1["atom_pos"], a0["atom_pos"])
    assert np.max(np.abs(a1["water_pos"] - a0["water_pos"])) > 1e-3
    st.step(0.002, 10)
    assert np.max(np.abs(st.state()["atom_pos"] - a1["atom_pos"])) > 1e-4
    st.close()


@pytest.mark.parametrize("lam", [0.25, 0.75])
@pytest.mark.parametrize("mode", ["reference", "corrected"])
def test_alchemical_forces_match_oracle(gpu_lib, relaxed, lam, mode):
    """The peptide decoupled at lambda (Coulomb stage, then soft-core LJ
    stage): forces, potential energy and dH/dlambda against the oracle."""
    n_pep = int(np.max(relaxed["bonds"])) + 1
    cfg = _cfg(relaxed, mode, alch_range=(0, n_pep), alch_lambda=lam)
    st = md.MdState(relaxed, cfg)
    got = st.forces()
    ref = method_alch(relaxed, cfg, st)
    err = _compare(got, ref)
    assert err < FORCE_RTOL, f"force rel-RMS {err:.3e}"
    assert abs(got["potential"] - ref["pe"]) <= PE_RTOL * abs(ref["pe"]), (got["potential"], ref["pe"])
    assert abs(got["dh_dl"] - ref["dh_dl"]) <= 1e-4 * max(1.0, abs(ref["dh_dl"])), (got["dh_dl"], ref["dh_dl"])
    # another window through set_lambda
    st.set_lambda(1.0 - lam)
    got2 = st.forces()
    cfg2 = _cfg(relaxed, mode, alch_range=(0, n_pep), alch_lambda=1.0 - lam)
    ref2 = method_alch(relaxed, cfg2, st)
    assert _compare(got2, ref2) < FORCE_RTOL
    assert abs(got2["dh_dl"] - ref2["dh_dl"]) <= 1e-4 * max(1.0, abs(ref2["dh_dl"]))
    st.close()


def method_alch(sysd, cfg, st):
    from oracle import method
    d = {**sysd, "water_m": st.state()["water_m"]}
    return method.all_forces(d, {
        "cutoff": cfg.coulomb_cutoff, "lj_cutoff": cfg.lj_cutoff, "alpha": float(np.float32(cfg.spme_alpha)),
        "grid": cfg.spme_grid, "mode": "corrected" if cfg.ewald_corrections else "reference",
        "alch_range": cfg.alch_range, "alch_lambda": float(np.float32(cfg.alch_lambda))})
