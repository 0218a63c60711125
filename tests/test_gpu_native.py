"""Parity of the device-resident engine (dyn_sys_*) with the float64 oracle.

Force evaluations are compared with oracle.method.all_forces, which finds
every site pair within the cutoff with a periodic k-d tree (independent of
any neighbour list), so a missing cluster pair or a wrong exclusion shows
up as a force error.  Tolerances are the ones the engine is specified to:
per-atom force relative RMS <= 1e-5 vs float64 (precision form), and
potential energy relative error <= 1e-6.
"""
import numpy as np
import pytest

from dynamics_b200 import md, synth
from oracle import integrate as oint
from oracle import method

from .systems import mixed, rel_rms, water_only

pytestmark = pytest.mark.gpu

FORCE_RTOL = 1e-5
PE_RTOL = 1e-6


def _cfg(sysd, mode="reference", integ=None, **kw):
    grid = kw.pop("spme_grid", None) or tuple(int(2 ** np.ceil(np.log2(x))) if x <= 32 else int(np.ceil(x / 8) * 8)
                                             for x in (sysd["box_hi"] - sysd["box_lo"]))
    c = md.MdConfig(coulomb_cutoff=8.0, lj_cutoff=8.0, spme_alpha=synth.ewald_alpha(8.0),
                    spme_grid=grid, ewald_corrections=(mode == "corrected"),
                    full_energy=(mode == "corrected"), **kw)
    if integ is not None:
        c.integrator = integ
    return c


def _oracle(sysd, cfg, st=None):
    """FP64 forces and energies of the kernel's own FP32 site coordinates:
    with ``st`` the M sites are the engine's (its float32 virtual-site
    placement), so both evaluate exactly the same coordinates."""
    if st is not None:
        sysd = {**sysd, "water_m": st.state()["water_m"]}
    # the engine's parameters are float32: the oracle evaluates the same values
    return method.all_forces(sysd, {
        "cutoff": cfg.coulomb_cutoff, "lj_cutoff": cfg.lj_cutoff, "alpha": float(np.float32(cfg.spme_alpha)),
        "grid": cfg.spme_grid, "mode": "corrected" if cfg.ewald_corrections else "reference"})


def _compare(got, ref):
    fa = np.concatenate([got["f_atoms"].reshape(-1), got["f_water"].reshape(-1)])
    fr = np.concatenate([ref["f_atoms"].reshape(-1), ref["f_water"].reshape(-1)])
    return rel_rms(fa, fr)


@pytest.mark.parametrize("mode", ["reference", "corrected"])
@pytest.mark.parametrize("make", [water_only, mixed])
def test_forces_match_oracle(gpu_lib, make, mode):
    sysd = make()
    cfg = _cfg(sysd, mode)
    st = md.MdState(sysd, cfg)
    got = st.forces()
    ref = _oracle(sysd, cfg, st)
    err = _compare(got, ref)
    assert err < FORCE_RTOL, f"force rel-RMS {err:.3e}"
    assert abs(got["potential"] - ref["pe"]) <= PE_RTOL * abs(ref["pe"]), (got["potential"], ref["pe"])
    assert abs(got["e_recip"] - ref["e_recip"]) <= 1e-6 * abs(ref["e_recip"])
    st.close()


def test_config1_forces_match_oracle(gpu_lib):
    sysd = synth.config1()
    cfg = md.MdConfig(coulomb_cutoff=10.0, lj_cutoff=10.0, spme_alpha=synth.ewald_alpha(10.0),
                      spme_grid=(32, 32, 32))
    st = md.MdState(sysd, cfg)
    got = st.forces()
    ref = _oracle(sysd, cfg)
    err = _compare(got, ref)
    assert err < FORCE_RTOL, f"force rel-RMS {err:.3e}"
    st.close()


@pytest.mark.parametrize("mode", ["reference", "corrected"])
def test_atoms_only_system(gpu_lib, mode):
    """A system without water (solute atoms only): forces and PE match the
    oracle, and the step graph runs with every water kernel skipped."""
    sysd = dict(mixed())
    sysd["water_pos"] = np.zeros((0, 3, 3), np.float32)
    sysd["water_vel"] = np.zeros((0, 3, 3), np.float32)
    cfg = _cfg(sysd, mode, integ=md.VerletVelocity(thermostat=None))
    st = md.MdState(sysd, cfg)
    got = st.forces()
    ref = _oracle(sysd, cfg, st)
    assert got["f_water"].shape == (0, 4, 3)
    err = _compare(got, ref)
    # With the Ewald corrections and no solvent, the float32 reciprocal
    # forces between bonded atoms nearly cancel against their FP64 exclusion
    # corrections, so the net forces of these 30 atoms are small next to the
    # rounding of their parts (1.1e-5 measured); with solvent the same
    # corrections stay within 1e-5 (5.3e-6 at 100k sites).
    tol = FORCE_RTOL if mode == "reference" else 2e-5
    assert err < tol, f"force rel-RMS {err:.3e}"
    assert abs(got["potential"] - ref["pe"]) <= PE_RTOL * abs(ref["pe"]), (got["potential"], ref["pe"])
    st.step(0.001, 20)
    e = st.energies()
    assert e["step"] == 20 and np.isfinite(e["potential"]) and np.isfinite(e["kinetic"])
    assert np.all(np.isfinite(st.state()["atom_pos"]))
    st.close()


def test_forces_deterministic(gpu_lib):
    sysd = mixed()
    cfg = _cfg(sysd)
    a = md.MdState(sysd, cfg)
    b = md.MdState(sysd, cfg)
    fa, fb = a.forces(), b.forces()
    np.testing.assert_array_equal(fa["f_water"], fb["f_water"])
    np.testing.assert_array_equal(fa["f_atoms"], fb["f_atoms"])
    a.step(0.002, 20)
    b.step(0.002, 20)
    sa, sb = a.state(), b.state()
    for k in sa:
        np.testing.assert_array_equal(sa[k], sb[k])
    a.close()
    b.close()


def _oracle_vv(sysd, cfg, n, dt):
    """n velocity-Verlet steps without thermostat in float64, SPME every step."""
    s = {
        "atom_pos": sysd["atom_pos"].astype(np.float64), "atom_vel": sysd["atom_vel"].astype(np.float64),
        "atom_mass": sysd["atom_mass"].astype(np.float64),
        "atom_static": np.zeros(len(sysd["atom_pos"]), bool),
        "water_pos": sysd["water_pos"].astype(np.float64), "water_vel": sysd["water_vel"].astype(np.float64),
    }
    lo = sysd["box_lo"].astype(np.float64)
    ext = (sysd["box_hi"] - sysd["box_lo"]).astype(np.float64)

    def forces(s):
        d = dict(sysd)
        d["atom_pos"] = s["atom_pos"]
        d["water_pos"] = s["water_pos"]
        d.pop("water_m", None)
        return _oracle(d, cfg)

    f = forces(s)
    oint.kick_and_calc_accel(s, f, 0.0)
    for _ in range(n):
        oint.kick_and_drift(s, dt / 2, dt, lo, ext)
        f = forces(s)
        oint.kick_and_calc_accel(s, f, dt / 2)
    return s


def test_short_trajectory_matches_oracle(gpu_lib):
    sysd = water_only()
    cfg = _cfg(sysd, integ=md.VerletVelocity(thermostat=None), spme_interval=1,
               zero_com_drift=False, recenter_sim_box=False)
    st = md.MdState(sysd, cfg)
    st.step(0.002, 5)
    got = st.state()
    ref = _oracle_vv(sysd, cfg, 5, 0.002)
    d = got["water_pos"].astype(np.float64) - ref["water_pos"]
    box = float(sysd["box_hi"][0] - sysd["box_lo"][0])
    d -= np.round(d / box) * box
    assert np.max(np.abs(d)) < 1e-4
    assert rel_rms(got["water_vel"], ref["water_vel"]) < 1e-4
    st.close()


def test_nve_energy_conservation(gpu_lib):
    sysd = water_only()
    cfg = _cfg(sysd, "corrected", integ=md.VerletVelocity(thermostat=None), spme_interval=1,
               zero_com_drift=False, recenter_sim_box=False, reset_angle=False)
    cfg.spme_grid = (32, 32, 32)
    sysd = md.equilibrate(sysd, cfg, n_steps=1000)
    st = md.MdState(sysd, cfg)
    e = []
    for _ in range(20):
        st.step(0.001, 10)
        en = st.energies()
        e.append(en["kinetic"] + en["potential"])
    e = np.array(e)
    drift = abs(e[-1] - e[0])
    assert drift < 2e-3 * abs(e[0]), (e[0], e[-1])
    st.close()


def test_langevin_thermalises(gpu_lib):
    sysd = synth.config1()
    cfg = md.MdConfig(coulomb_cutoff=10.0, lj_cutoff=10.0, spme_alpha=synth.ewald_alpha(10.0),
                      spme_grid=(32, 32, 32), integrator=md.LangevinMiddle(gamma=1.0), seed=7)
    sysd = md.equilibrate(sysd, cfg, n_steps=1000)
    st = md.MdState(sysd, cfg)
    st.step(0.002, 200)
    en = st.energies()
    assert np.isfinite(en["potential"]) and 200.0 < en["temperature"] < 400.0
    assert en["list_rebuilds"] >= 1
    st.close()


def test_csvr_holds_temperature(gpu_lib):
    sysd = mixed()
    cfg = _cfg(sysd, integ=md.VerletVelocity(thermostat=0.1), seed=3)
    sysd = md.equilibrate(sysd, cfg, n_steps=1000)
    st = md.MdState(sysd, cfg)
    st.step(0.001, 300)
    en = st.energies()
    assert 220.0 < en["temperature"] < 380.0
    st.close()


def test_invalid_config_raises(gpu_lib):
    from dynamics_b200 import DynError
    sysd = water_only(n_side=3)
    with pytest.raises(DynError):
        md.MdState(sysd, md.MdConfig(coulomb_cutoff=10.0))  # box too small for the cutoff


def test_union_chunking(gpu_lib):
    """The water-water kernel stages a group's j-waters in shared-memory
    chunks, and its threads' shares of the list entries follow the chunks,
    so a different chunk size groups the float i-force sums differently:
    forces agree to rounding, and every chunk size is bit-identical run to
    run."""
    sysd = water_only()
    a = md.MdState(sysd, _cfg(sysd))
    b = md.MdState(sysd, _cfg(sysd, ww_union_chunk=64))
    b2 = md.MdState(sysd, _cfg(sysd, ww_union_chunk=64))
    fa, fb, fb2 = a.forces(), b.forces(), b2.forces()
    assert rel_rms(fb["f_water"].reshape(-1), fa["f_water"].reshape(-1)) < 1e-6
    assert abs(fa["virial"] - fb["virial"]) <= 1e-6 * abs(fa["virial"])
    np.testing.assert_array_equal(fb["f_water"], fb2["f_water"])
    a.step(0.002, 30)
    b.step(0.002, 30)
    b2.step(0.002, 30)
    sb = b.state()
    np.testing.assert_array_equal(sb["water_pos"], b2.state()["water_pos"])
    assert np.max(np.abs(sb["water_pos"] - a.state()["water_pos"])) < 1e-3
    assert a.energies()["list_union_max"] > 64
    for st in (a, b, b2):
        st.close()


@pytest.mark.parametrize("grid", [None, (25, 27, 33)])
@pytest.mark.parametrize("mode", ["reference", "corrected"])
@pytest.mark.parametrize("make", [water_only, mixed])
def test_spme_bricks_bit_identical_to_per_site(gpu_lib, make, mode, grid):
    """SPME spreads and gathers by grid brick in shared memory; with a brick
    capacity of 1 nearly every charged site takes the overflow path (global
    fixed-point atomics, per-site gather from the global grid, the per-site
    arithmetic).  Forces, the reciprocal energy and the trajectory must be
    the same bits either way.  Grid 25 x 27 x 33 has axes whose last brick
    is narrower than 3 points, where the spread's second phase takes its
    per-point form."""
    sysd = make()
    kw = {"spme_grid": grid} if grid else {}
    a = md.MdState(sysd, _cfg(sysd, mode, **kw))
    b = md.MdState(sysd, _cfg(sysd, mode, spme_brick_cap=1, **kw))
    fa, fb = a.forces(), b.forces()
    np.testing.assert_array_equal(fa["f_water"], fb["f_water"])
    np.testing.assert_array_equal(fa["f_atoms"], fb["f_atoms"])
    assert fa["e_recip"] == fb["e_recip"] and fa["virial_recip"] == fb["virial_recip"]
    a.step(0.002, 20)
    b.step(0.002, 20)
    sa, sb = a.state(), b.state()
    for k in sa:
        np.testing.assert_array_equal(sa[k], sb[k], err_msg=k)
    a.close()
    b.close()


def test_snapshot_memory_handler(gpu_lib):
    """MdConfig.snapshot_memory (SnapshotHandlers.memory) records a frame
    every N steps; MdState.snapshots returns them as Snapshot objects with
    the reference's field names, accumulating across reads."""
    sysd = mixed()
    cfg = _cfg(sysd, integ=md.LangevinMiddle(gamma=1.0), seed=3, snapshot_memory=4)
    st = md.MdState(sysd, cfg)
    st.step(0.002, 8)
    s8 = st.state()
    snaps = st.snapshots
    assert [x.step for x in snaps] == [4, 8]
    st.step(0.002, 4)
    snaps = st.snapshots
    assert [x.step for x in snaps] == [4, 8, 12]
    x = snaps[1]
    nw, na = len(s8["water_pos"]), len(s8["atom_pos"])
    np.testing.assert_array_equal(x.water_o_posits, s8["water_pos"][:, 0])
    np.testing.assert_array_equal(x.water_h1_posits, s8["water_pos"][:, 2])
    np.testing.assert_array_equal(x.water_velocities, s8["water_vel"][:, 0])
    np.testing.assert_array_equal(x.atom_velocities, s8["atom_vel"])
    assert x.atom_posits.shape == (na, 3) and x.water_h0_posits.shape == (nw, 3)
    assert abs(x.time - float(np.float32(0.002)) * 8) < 1e-9
    e = x.energy_data
    assert e.temperature > 0 and e.volume > 0 and e.density > 0 and e.dh_dl is None
    assert abs(e.energy_potential_nonbonded + e.energy_potential_bonded - e.energy_potential) < 1e-6
    assert "MdState" in str(st)
    st.close()


def test_graph_counters_and_periodic_tasks(gpu_lib):
    """Steps run as captured graphs whose list rebuild and periodic tasks
    are conditional nodes set on the device: the step counter, the rebuild
    count and the COM removal at step 100 must all happen."""
    sysd = md.equilibrate(mixed(), _cfg(mixed()), n_steps=50, dt=0.001)
    cfg = _cfg(sysd, integ=md.LangevinMiddle(gamma=5.0), com_removal_interval=100)
    st = md.MdState(sysd, cfg)
    st.step(0.002, 100)
    e = st.energies()
    assert e["step"] == 100
    assert e["list_rebuilds"] >= 1
    s = st.state()
    m_w = np.array([16.0, 1.008, 1.008])  # site masses the engine uses
    p = (s["water_vel"] * m_w[None, :, None]).sum(axis=(0, 1))
    p += (s["atom_vel"] * np.asarray(sysd["atom_mass"])[:, None]).sum(axis=0)
    p_scale = np.abs(s["water_vel"] * m_w[None, :, None]).sum()
    assert np.linalg.norm(p) < 1e-4 * p_scale, (p, p_scale)
    st.step(0.002, 7)
    assert st.energies()["step"] == 107
    st.close()


def test_snapshots_match_state(gpu_lib):
    """Frames recorded by the step graph equal the state read back at the
    same steps; frames that overflow the ring are counted as lost."""
    sysd = mixed()
    cfg = _cfg(sysd, integ=md.LangevinMiddle(gamma=1.0), seed=5)
    st = md.MdState(sysd, cfg)
    st.enable_snapshots(ratio=5, capacity=4, velocities=True, forces=True)
    ref = []
    for _ in range(3):
        st.step(0.002, 5)
        s = st.state()
        ref.append(s)
    frames = st.read_snapshots()
    assert [f["step"] for f in frames] == [5, 10, 15]
    lo = sysd["box_lo"].astype(np.float64)
    ext = (sysd["box_hi"] - sysd["box_lo"]).astype(np.float64)
    for f, s in zip(frames, ref):
        na = len(s["atom_pos"])
        wrapped = s["atom_pos"] - np.floor((s["atom_pos"] - lo) / ext) * ext
        np.testing.assert_allclose(f["pos"][:na], wrapped, atol=1e-4)
        np.testing.assert_array_equal(f["pos"][na:], s["water_pos"].reshape(-1, 3))
        np.testing.assert_array_equal(f["vel"][:na], s["atom_vel"])
        np.testing.assert_array_equal(f["vel"][na:], s["water_vel"].reshape(-1, 3))
        assert f["force"].shape == (na, 3) and np.all(np.isfinite(f["force"]))
        # time is the sum of the float32 step lengths
        assert abs(f["time_ps"] - float(np.float32(0.002)) * f["step"]) < 1e-9
        assert f["volume"] > 0 and f["density"] > 0
    assert frames[0]["lost"] == 0
    st.step(0.002, 30)  # 6 frames into a ring of 4
    more = st.read_snapshots()
    assert [f["step"] for f in more] == [30, 35, 40, 45] and more[0]["lost"] == 2
    st.enable_snapshots(0)
    st.step(0.002, 5)
    assert st.read_snapshots() == []
    st.close()
