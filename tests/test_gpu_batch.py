"""The batched form (dyn_batch_*): systems of different sizes advanced in
one launch per stage must give exactly the trajectories they give alone.

Every force is accumulated as 64-bit fixed point and every stochastic term
is keyed by (site, step, seed), so "the same" means bit-identical positions,
velocities and energies, not a tolerance.
"""
import numpy as np
import pytest

from dynamics_b200 import md, peptide, synth

from .systems import mixed, water_only

pytestmark = pytest.mark.gpu


def _cfg(sysd, integ=None, **kw):
    box = float(sysd["box_hi"][0] - sysd["box_lo"][0])
    k = synth.fft_size(int(np.ceil(box)))
    # ww_split 1: what a batch member gets by default, so the same system
    # alone runs the same water-water partition
    kw.setdefault("ww_split", 1)
    c = md.MdConfig(coulomb_cutoff=8.0, lj_cutoff=8.0, spme_alpha=synth.ewald_alpha(8.0),
                    spme_grid=(k, k, k), **kw)
    if integ is not None:
        c.integrator = integ
    return c


def _members():
    # the last member: a ten-residue peptide with counter-ions and
    # bond-to-hydrogen constraints
    pep, _, _ = peptide.batch_member(600, 1, seed=6)
    systems = [water_only(n_side=7, seed=3), synth.water_box(512, 24.8, seed=4),
               synth.water_box(729, 27.9, seed=5), mixed(), pep]
    cfgs = [
        _cfg(systems[0], integ=md.LangevinMiddle(gamma=1.0), seed=11),
        _cfg(systems[1], integ=md.VerletVelocity(thermostat=0.1), seed=12),
        _cfg(systems[2], integ=md.VerletVelocity(thermostat=0.1), seed=13,
             barostat_cfg=md.BarostatCfg()),
        _cfg(systems[3], integ=md.LangevinMiddle(gamma=1.0), seed=14),
        _cfg(systems[4], integ=md.LangevinMiddle(gamma=1.0), seed=15),
    ]
    systems = [md.equilibrate(s, c, n_steps=40, dt=0.001) for s, c in zip(systems, cfgs)]
    return systems, cfgs


def test_batch_matches_members_alone(gpu_lib):
    systems, cfgs = _members()
    n_steps = 60  # crosses list rebuilds, SPME and non-SPME steps
    batch = md.MdBatch(systems, cfgs)
    batch.step(0.002, n_steps)
    batch.sync()
    for i, (s, c) in enumerate(zip(systems, cfgs)):
        alone = md.MdState(s, c)
        alone.step(0.002, n_steps)
        a, b = alone.state(), batch.members[i].state()
        for k in a:
            np.testing.assert_array_equal(a[k], b[k], err_msg=f"member {i} {k}")
        ea, eb = alone.energies(), batch.members[i].energies()
        for k in ("potential", "kinetic", "virial", "temperature", "pressure_bar", "step", "list_rebuilds"):
            assert ea[k] == eb[k], (i, k, ea[k], eb[k])
        alone.close()
    batch.close()


def test_batch_is_one_launch_per_stage(gpu_lib):
    systems, cfgs = _members()
    batch = md.MdBatch(systems, cfgs)
    fixed, rebuild, periodic = batch.launches(spme=True)
    per_system = [md.MdState(s, c) for s, c in zip(systems, cfgs)]
    plain = sum(p.launches_per_step(True) for p in per_system)
    # one launch per stage for all members, against one per stage per member
    assert fixed < plain / 2, (fixed, plain)
    assert fixed <= max(p.launches_per_step(True) for p in per_system) + 2
    assert rebuild > 0 and periodic > 0
    for p in per_system:
        p.close()
    batch.close()


def test_batch_rejects_mixed_intervals(gpu_lib):
    systems, cfgs = _members()
    cfgs[1] = _cfg(systems[1], spme_interval=1)
    with pytest.raises(Exception):
        md.MdBatch(systems[:2], cfgs[:2])


def test_batch_host_step_matches_members_host_step(gpu_lib):
    """dyn_batch_step_host (one copy each way for the whole batch) gives
    each member exactly what dyn_sys_step_host gives it alone on the same
    host state, and reads back the states dyn_sys_get_state reads."""
    systems, cfgs = _members()
    batch = md.MdBatch(systems, cfgs)
    buf = batch.host_buffer()
    off = batch.state_layout()
    assert len(buf) == off[-1] and len(off) == len(systems) + 1
    # the resident states, read back through the packed path
    batch.step_host(0.002, 3, None, buf)
    for i, m in enumerate(batch.members):
        s, v = m.state(), batch.unpack(buf, i)
        for k in v:
            np.testing.assert_array_equal(np.asarray(s[k], np.float32).reshape(v[k].shape), v[k],
                                          err_msg=f"member {i} {k}")
    host_in = buf.copy()
    alone = []
    for i, (s, c) in enumerate(zip(systems, cfgs)):
        st = md.MdState(s, c)
        st.step(0.002, 3)
        io = {k: np.ascontiguousarray(a) for k, a in batch.unpack(host_in.copy(), i).items()}
        e = st.step_host(0.002, 20, io, io)
        alone.append((io, e))
        st.close()
    en = batch.step_host(0.002, 20, buf, buf, energies=True)
    for i, (io, e) in enumerate(alone):
        v = batch.unpack(buf, i)
        for k in v:
            np.testing.assert_array_equal(io[k], v[k], err_msg=f"member {i} {k}")
        for k in ("potential", "kinetic", "virial", "temperature", "step", "list_rebuilds"):
            assert e[k] == en[i][k], (i, k, e[k], en[i][k])
    batch.close()
