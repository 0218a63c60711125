"""The autotuner on the device: it picks run-time knobs by timing real steps,
caches the choice by size class (a second call returns it without timing),
and a tuned configuration computes the same method: forces within the
engine's tolerance of the float64 oracle.  A batch built with tune=True
steps its members with their classes' choices, each bit-identical to the
same member run alone with that configuration."""
import numpy as np
import pytest

from dynamics_b200 import md, synth, tune
from oracle import method

from .systems import rel_rms

pytestmark = pytest.mark.gpu


def _sys(n, seed):
    sysd, grid = synth.batch_member(n, seed=seed)
    cfg = md.MdConfig(coulomb_cutoff=9.0, lj_cutoff=9.0, spme_alpha=synth.ewald_alpha(9.0), spme_grid=grid, ww_split=1,
                      integrator=md.LangevinMiddle(gamma=1.0), seed=seed)
    return sysd, cfg


def test_tune_caches_and_keeps_accuracy(gpu_lib, tmp_path, monkeypatch):
    monkeypatch.setenv("DYNB200_TUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(tune, "SHIPPED", str(tmp_path / "none.json"))
    sysd, cfg = _sys(700, 3)
    knobs = tune.tune(sysd, cfg, steps=20, warmup=5)
    assert set(knobs) == set(tune.KNOBS)
    calls = []
    monkeypatch.setattr(tune, "time_steps", lambda *a, **k: calls.append(1) or 1.0)
    assert tune.tune(sysd, cfg) == knobs and not calls  # from the cache
    tuned = tune.apply_tuned(sysd, cfg)
    st = md.MdState(sysd, tuned)
    got = st.forces()
    m = st.state()["water_m"]
    st.close()
    ref = method.all_forces({**sysd, "water_m": m}, {
        "cutoff": 9.0, "lj_cutoff": 9.0, "alpha": float(np.float32(cfg.spme_alpha)), "grid": tuned.spme_grid,
        "mode": "reference"})
    assert rel_rms(got["f_water"].reshape(-1), ref["f_water"].reshape(-1)) < 1e-5


def test_tuned_batch_members_equal_alone(gpu_lib, tmp_path, monkeypatch):
    monkeypatch.setenv("DYNB200_TUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(tune, "SHIPPED", str(tmp_path / "none.json"))
    systems, cfgs = zip(*[_sys(n, 10 + i) for i, n in enumerate((600, 1500))])
    monkeypatch.setattr(tune, "time_steps", lambda system, cfg, *a, **k: 1.0 + 0.1 * cfg.neighbor_skin)
    b = md.MdBatch(systems, cfgs, tune=True)
    b.step(0.002, 10)
    b.sync()
    for i, (sysd, c) in enumerate(zip(systems, b.cfgs)):
        assert c.neighbor_skin == min(tune.SKINS)  # the fake timings favour the smallest buffer
        alone = md.MdState(sysd, c)
        alone.step(0.002, 10)
        sa, sb = alone.state(), b.members[i].state()
        np.testing.assert_array_equal(sa["water_pos"], sb["water_pos"])
        alone.close()
    b.close()
