"""Host logic of MdState.snapshots: frames as read from the device ring
become Snapshot / SnapshotEnergyData objects with the reference's field
names (src/snapshot.rs:61-175), accumulating across reads.  The device read
is replaced by synthetic frames, so this runs without a GPU."""
import numpy as np

from dynamics_b200 import md


def _frame(step, na, nw, rng, with_vel):
    pos = rng.normal(size=(na + 3 * nw, 3)).astype(np.float32)
    d = {"step": step, "time_ps": 0.002 * step, "kinetic": 10.0 + step, "potential": -50.0 - step,
         "potential_bonded": 4.0, "temperature": 300.0, "pressure_bar": 1.5,
         "box_lo": [0.0, 0.0, 0.0], "box_hi": [20.0, 21.0, 22.0], "volume": 9240.0,
         "density": 0.6, "dh_dl": 3.25, "pos": pos}
    if with_vel:
        d["vel"] = rng.normal(size=pos.shape).astype(np.float32)
    return d


def _state(na, nw, cfg):
    st = md.MdState.__new__(md.MdState)
    st.n_atoms, st.n_water, st.cfg = na, nw, cfg
    st._snapshots = []
    return st


def test_snapshot_fields_and_accumulation():
    rng = np.random.default_rng(0)
    na, nw = 5, 4
    st = _state(na, nw, md.MdConfig())
    batches = [[_frame(10, na, nw, rng, True), _frame(20, na, nw, rng, True)], [_frame(30, na, nw, rng, True)], []]
    st.read_snapshots = lambda: batches.pop(0)
    first = st.snapshots
    assert [x.step for x in first] == [10, 20]
    again = st.snapshots
    assert [x.step for x in again] == [10, 20, 30]
    assert [x.step for x in st.snapshots] == [10, 20, 30]
    x = again[2]
    assert x.atom_posits.shape == (na, 3)
    for arr in (x.water_o_posits, x.water_h0_posits, x.water_h1_posits, x.water_velocities):
        assert arr.shape == (nw, 3)
    e = x.energy_data
    assert e.energy_potential == -80.0 and e.energy_potential_bonded == 4.0
    assert e.energy_potential_nonbonded == -84.0
    assert e.pressure == 1.5 and e.temperature == 300.0 and e.dh_dl is None
    assert x.cell == ((0.0, 0.0, 0.0), (20.0, 21.0, 22.0))
    assert abs(x.time - 0.06) < 1e-12


def test_snapshot_site_layout_and_alchemical_dhdl():
    rng = np.random.default_rng(1)
    na, nw = 3, 2
    st = _state(na, nw, md.MdConfig(alch_range=(0, 3), alch_lambda=0.5))
    fr = _frame(5, na, nw, rng, False)
    st.read_snapshots = lambda: [fr]
    (x,) = st.snapshots
    w = fr["pos"][na:].reshape(nw, 3, 3)
    np.testing.assert_array_equal(x.water_o_posits, w[:, 0])
    np.testing.assert_array_equal(x.water_h0_posits, w[:, 1])
    np.testing.assert_array_equal(x.water_h1_posits, w[:, 2])
    assert x.atom_velocities is None and x.water_velocities is None and x.force is None
    assert x.energy_data.dh_dl == 3.25
