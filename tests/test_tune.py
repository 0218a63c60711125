"""The autotuner's host logic: size classes, grid candidates (never coarser
than the configured spacing), the tie rule that keeps a choice stable under
timing noise, and the cache round trip (no GPU needed)."""
import numpy as np

from dynamics_b200 import md, synth, tune


def _cfg(grid):
    return md.MdConfig(coulomb_cutoff=9.0, lj_cutoff=9.0, spme_alpha=synth.ewald_alpha(9.0), spme_grid=grid)


def test_size_class_groups_similar_systems():
    a = synth.water_box(1000, 31.0, seed=1)
    b = synth.water_box(1050, 31.5, seed=2)
    c = synth.water_box(4000, 49.2, seed=3)
    assert tune.size_class(a, _cfg((32, 32, 32))) == tune.size_class(b, _cfg((32, 32, 32)))
    assert tune.size_class(a, _cfg((32, 32, 32))) != tune.size_class(c, _cfg((50, 50, 50)))


def test_grid_candidates_hold_the_spacing():
    sysd = synth.water_box(1000, 31.0, seed=1)
    base = (32, 32, 32)
    cands = tune.grid_candidates(sysd, _cfg(base))
    assert cands[0] == base and len(cands) >= 2
    spacing = 31.0 / 32
    for g in cands:
        assert all(31.0 / k <= spacing + 1e-9 for k in g), g
        assert all(synth.fft_size(k) == k for k in g), g


def test_pick_is_stable_under_noise():
    order = [1.5, 1.0, 1.25, 1.75]
    # the incumbent (first in order) stays unless something is clearly faster
    assert tune.pick({1.5: 1.00, 1.0: 0.99, 1.25: 1.01, 1.75: 1.05}, order) == 1.5
    assert tune.pick({1.5: 1.00, 1.0: 0.90, 1.25: 1.01, 1.75: 1.05}, order) == 1.0
    # ties beyond the incumbent go to the earlier candidate
    assert tune.pick({1.5: 1.10, 1.0: 0.99, 1.25: 1.00, 1.75: 1.2}, order) == 1.0


def test_cache_round_trip(tmp_path, monkeypatch):
    monkeypatch.setenv("DYNB200_TUNE_CACHE", str(tmp_path / "t.json"))
    monkeypatch.setattr(tune, "SHIPPED", str(tmp_path / "none.json"))
    sysd = synth.water_box(1000, 31.0, seed=1)
    cfg = _cfg((32, 32, 32))
    key = tune.size_class(sysd, cfg)
    knobs = {"neighbor_skin": 1.25, "prune_buffer": 0.3, "ww_union_chunk": 0, "spme_grid_step": 1}
    tune.save_cache({key: {"knobs": knobs}})
    got = tune.apply_tuned(sysd, cfg)
    assert got.neighbor_skin == 1.25 and got.prune_buffer == 0.3
    assert got.spme_grid == tune.grid_candidates(sysd, cfg)[1]
    assert tune.tune(sysd, cfg) == knobs
    # a class member with a finer configured grid keeps a grid at least as fine
    same_class = synth.water_box(1050, 31.5, seed=2)
    assert tune.size_class(same_class, _cfg((36, 36, 36))) == key
    g = tune.apply_tuned(same_class, _cfg((36, 36, 36))).spme_grid
    assert all(31.5 / k <= 31.5 / 36 + 1e-9 for k in g)
    other = synth.water_box(4000, 49.2, seed=3)
    assert tune.apply_tuned(other, _cfg((50, 50, 50))).spme_grid == (50, 50, 50)


def test_shipped_table_behind_user_cache(tmp_path, monkeypatch):
    """A class missing from the user's cache comes from the shipped table;
    the user's cache wins where both have it."""
    import json
    monkeypatch.setenv("DYNB200_TUNE_CACHE", str(tmp_path / "t.json"))
    shipped = tmp_path / "shipped.json"
    monkeypatch.setattr(tune, "SHIPPED", str(shipped))
    sysd = synth.water_box(1000, 31.0, seed=1)
    cfg = _cfg((32, 32, 32))
    key = tune.size_class(sysd, cfg)
    assert tune.lookup(key) is None
    ship = {"neighbor_skin": 1.75, "prune_buffer": 0.6, "ww_union_chunk": 0, "spme_grid_step": 0}
    shipped.write_text(json.dumps({key: {"knobs": ship}}))
    assert tune.lookup(key) == ship
    assert tune.apply_tuned(sysd, cfg).neighbor_skin == 1.75
    mine = dict(ship, neighbor_skin=1.25)
    tune.save_cache({key: {"knobs": mine}})
    assert tune.lookup(key) == mine and tune.tune(sysd, cfg) == mine
