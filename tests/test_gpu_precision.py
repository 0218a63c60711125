"""Precision form at config-3 size: a 300-residue ff19SB peptide with 0.15 M
NaCl and counter-ions in 23,822 OPC waters (100,311 sites, 98 A box, rc 10,
SPME 96^3).  Forces and potential energy are compared with the float64
oracle (per-site force relative RMS <= 1e-5, potential energy relative
error <= 1e-6), and the total energy of a 100 ps constant-energy run is
fitted for its drift per ns and per atom."""
import json
import os

import numpy as np
import pytest

from dynamics_b200 import md, peptide, synth

from .test_gpu_native import FORCE_RTOL, PE_RTOL, _compare, _oracle

pytestmark = pytest.mark.gpu

# records of the precision runs go to the directory named by DYNB200_OUT
OUT = os.environ.get("DYNB200_OUT", "")


def _cfg(**kw):
    return md.MdConfig(coulomb_cutoff=10.0, lj_cutoff=10.0, spme_alpha=synth.ewald_alpha(10.0),
                       spme_grid=(96, 96, 96), seed=1000, **kw)


def _report(name, rec):
    print(name, json.dumps(rec))
    if OUT and os.path.isdir(OUT):
        with open(os.path.join(OUT, f"precision_{name}.json"), "w") as f:
            json.dump(rec, f)


@pytest.fixture(scope="module")
def c3():
    sysd, _ = peptide.solvated_system(98.0, 24000, n_res=(300,), seed=1000, nacl_molar=0.15)
    cfg = _cfg(integrator=md.VerletVelocity(thermostat=0.1))
    return md.equilibrate(sysd, cfg, n_steps=300, dt=0.001)


@pytest.mark.parametrize("mode", ["reference", "corrected"])
def test_c3_forces_match_oracle(gpu_lib, c3, mode):
    cfg = _cfg(ewald_corrections=(mode == "corrected"), full_energy=(mode == "corrected"))
    st = md.MdState(c3, cfg)
    got = st.forces()
    ref = _oracle(c3, cfg, st)
    err = _compare(got, ref)
    pe_err = abs(got["potential"] - ref["pe"]) / abs(ref["pe"])
    _report(f"c3_forces_{mode}", {"force_rel_rms": err, "pe_rel": pe_err, "pe": got["potential"],
                                  "pe_oracle": ref["pe"]})
    assert err < FORCE_RTOL, f"force rel-RMS {err:.3e}"
    assert pe_err <= PE_RTOL, (got["potential"], ref["pe"])
    st.close()


@pytest.mark.parametrize("rattle_velocities", [True, False])
def test_c3_nve_drift(gpu_lib, c3, rattle_velocities):
    """100 ps of velocity Verlet without thermostat or barostat, SPME every
    step (the cached reciprocal forces of the reference's every-2-steps
    schedule are not a conservative force), full energy with the Ewald
    corrections; drift = slope of a linear fit of the total energy.  With
    the reference's position-only constraint correction the constrained
    bonds lose kinetic energy every step; that drift is reported, the
    energy-conserving variant's is held to a bound."""
    cfg = _cfg(integrator=md.VerletVelocity(thermostat=None), spme_interval=1, ewald_corrections=True,
               full_energy=True, zero_com_drift=False, recenter_sim_box=False, reset_angle=False,
               energy_interval=500, rattle_velocities=rattle_velocities)
    st = md.MdState(c3, cfg)
    dt, n_blocks, per = 0.002, 100, 500  # 100 x 500 steps of 2 fs = 100 ps
    t, e = [], []
    for k in range(n_blocks):
        st.step(dt, per)
        en = st.energies()
        t.append((k + 1) * per * dt)
        # the kinetic energy the rigid waters keep (rigid-body) + the atoms'
        e.append(en["kinetic_rigid"] + en["potential"])
    t, e = np.array(t), np.array(e)
    slope = np.polyfit(t, e, 1)[0]  # kcal/mol/ps
    n_atoms = 3 * len(c3["water_pos"]) + len(c3["atom_pos"])
    drift = slope * 1000.0 / n_atoms  # kcal/mol/ns/atom
    rec = {"drift_kcal_per_mol_ns_atom": drift, "e0": e[0], "e_end": e[-1], "e_std": float(np.std(e)),
           "ps": float(t[-1]), "atoms": n_atoms, "temperature_end": st.energies()["temperature"]}
    _report("c3_nve_" + ("rattle" if rattle_velocities else "reference"), rec)
    assert np.all(np.isfinite(e))
    if rattle_velocities:
        assert abs(drift) < 0.05, rec
    st.close()
