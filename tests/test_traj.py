"""Trajectory writers (DCD, TRR) on synthetic frames: byte layout of the
headers and round trips through the readers, with the unit conversions."""
import struct

import numpy as np

from dynamics_b200 import traj


def _frames(n_frames=3, n=7, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_frames):
        out.append({"step": 10 * (k + 1), "time_ps": 0.02 * (k + 1),
                    "pos": rng.uniform(0, 30, (n, 3)).astype(np.float32),
                    "vel": rng.normal(size=(n, 3)).astype(np.float32),
                    "force": rng.normal(size=(n, 3)).astype(np.float32),
                    "box_lo": [0.0, 0.0, 0.0], "box_hi": [30.0, 31.0, 32.0]})
    return out


def test_dcd_layout_and_round_trip(tmp_path):
    fr = _frames()
    p = tmp_path / "t.dcd"
    traj.write_dcd(p, fr, steps_between=10, dt_ps=0.002)
    raw = p.read_bytes()
    assert struct.unpack_from("<i", raw, 0)[0] == 84 and raw[4:8] == b"CORD"
    pos, cells, icntrl = traj.read_dcd(p)
    assert icntrl[0] == 3 and icntrl[1] == 10 and icntrl[2] == 10 and icntrl[10] == 1
    np.testing.assert_array_equal(pos, np.stack([f["pos"] for f in fr]))
    np.testing.assert_allclose(cells[:, [0, 2, 5]], [[30.0, 31.0, 32.0]] * 3)
    np.testing.assert_allclose(cells[:, [1, 3, 4]], 90.0)


def test_trr_round_trip_units(tmp_path):
    fr = _frames()
    p = tmp_path / "t.trr"
    traj.write_trr(p, fr[:2])
    traj.write_trr(p, fr[2:], append=True)
    raw = p.read_bytes()
    assert struct.unpack_from(">iii", raw, 0) == (1993, 13, 12) and raw[12:24] == b"GMX_trn_file"
    back = traj.read_trr(p)
    assert [b["step"] for b in back] == [10, 20, 30]
    for a, b in zip(fr, back):
        np.testing.assert_allclose(b["x"], a["pos"] * 0.1, rtol=1e-6)
        np.testing.assert_allclose(b["v"], a["vel"] * 0.1, rtol=1e-6)
        np.testing.assert_allclose(b["f"], a["force"] * 41.84, rtol=1e-6)
        np.testing.assert_allclose(np.diag(b["box"]), [3.0, 3.1, 3.2], rtol=1e-6)
        assert abs(b["time_ps"] - a["time_ps"]) < 1e-6


def test_trr_skips_partial_forces(tmp_path):
    fr = _frames(1)
    fr[0]["force"] = fr[0]["force"][:3]  # atoms only: not all sites
    p = tmp_path / "t.trr"
    traj.write_trr(p, fr)
    back = traj.read_trr(p)
    assert "f" not in back[0] and "v" in back[0]
