"""Autotuner for the resident engine's run-time parameters.

The engine's tile shapes are fixed at compile time (32-water groups, 8 lanes
per water, 8-body clusters); what varies per system is chosen here by
measurement, per size class of system, and cached:

* ``neighbor_skin``: the Verlet buffer of the cluster and molecule lists
  (longer lists against fewer rebuilds);
* ``prune_buffer``: the inner buffer of the pruned water-water lists
  (shorter lists against more prunes);
* ``ww_union_chunk``: the water-water kernel's shared-memory chunk (waters
  staged at a time; three CTAs per SM at the largest);
* ``pair_item_entries``: list entries per work item of the water-atom and
  atom-atom pair kernels (more items balance better, fewer amortise the
  per-item loads);
* ``ww_split``: CTAs sharing one water group's list entries (more CTAs
  shorten the last wave, each stages the group's union again);
* ``spme_grid``: the SPME grid among FFT-friendly sizes whose spacing is at
  most the configured grid's (the accuracy rule: a finer grid is never less
  accurate, so every candidate holds the force tolerance), at the
  reference's fixed spline order 4 (src/config.rs:208).  It is cached as a
  step in the system's own candidate list (0 = the configured grid), so a
  class member never gets a grid coarser than its configuration asks.

None of them changes the physics beyond the grid's (finer grids only
reduce the reciprocal-space error); the others change how float sums are
grouped, so results move only at rounding level: the same method within
the engine's force tolerance, and bit-identical run to run for a given
choice.  The search is coordinate descent from the
defaults: one knob at a time, each candidate timed over whole captured steps
(the step graph as MdState.step runs it), the fastest kept unless the
incumbent is within ``tie`` of it, so small timing noise does not flip a
choice.  Results are cached by size class in a JSON file
(``DYNB200_TUNE_CACHE``, default ~/.cache/dynb200/tune.json); classes
missing there are looked up in the table measured on B200 that ships with
the package (``data/tune_b200.json``) before anything is timed.  The
batched form (md.MdBatch(..., tune=True)) applies each member's class's
choice.

The reference has no tuner (its parameters are constants, src/config.rs);
this module is new.
"""
import dataclasses
import json
import math
import os
import time

import numpy as np

from . import md, synth

KNOBS = ("neighbor_skin", "prune_buffer", "ww_union_chunk", "ww_split", "pair_item_entries", "spme_grid_step")
SKINS = (1.0, 1.25, 1.5, 1.75, 2.0)
PRUNES = (0.2, 0.3, 0.4, 0.6, 0.8)
CHUNKS = (0, 256, 512)          # 0: the largest that lets three CTAs share an SM
ITEMS = (4, 8, 16, 32)
SPLITS = (0, 1, 2, 4)           # 0: automatic
GRID_SPAN = 1.15                # grid candidates up to 15 % above the finest needed


SHIPPED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "tune_b200.json")


def cache_path():
    return os.environ.get("DYNB200_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "dynb200",
                                                               "tune.json")


def size_class(system, cfg):
    """Key of the systems that share a tuning: water count in half-octaves,
    solute atoms in octaves, cutoff and integrator kind."""
    nw = len(np.asarray(system.get("water_pos", np.zeros((0, 3, 3)))).reshape(-1, 9))
    na = len(np.asarray(system.get("atom_pos", np.zeros((0, 3)))).reshape(-1, 3))
    cw = int(round(2.0 * math.log2(max(nw, 1))))
    ca = int(round(math.log2(na))) if na else -1
    return f"w{cw}_a{ca}_rc{cfg.coulomb_cutoff:g}_{type(cfg.integrator).__name__}"


def grid_candidates(system, cfg):
    """FFT-friendly grids (factors 2, 3, 5, 7) with a spacing no coarser than
    the configured grid's, up to GRID_SPAN above the finest needed per axis;
    the configured grid first."""
    ext = np.asarray(system["box_hi"], np.float64) - np.asarray(system["box_lo"], np.float64)
    base = tuple(int(k) for k in cfg.spme_grid)
    spacing = float(np.max(ext / np.asarray(base, np.float64)))
    need = [int(math.ceil(e / spacing - 1e-9)) for e in ext]
    out = [base]
    k = [synth.fft_size(n) for n in need]
    while True:
        cand = tuple(k)
        if all(c <= n * GRID_SPAN for c, n in zip(cand, need)) and cand not in out:
            out.append(cand)
        nxt = [synth.fft_size(c + 1) for c in k]
        if any(c > n * GRID_SPAN for c, n in zip(nxt, need)):
            break
        k = nxt
    return out


def pick(times, order, tie=0.02):
    """The candidate to keep: the fastest, unless the earliest candidate in
    ``order`` (the incumbent first) is within ``tie`` of it.  ``times`` maps
    candidate -> seconds per step."""
    best = min(times.values())
    for c in order:
        if c in times and times[c] <= best * (1.0 + tie):
            return c
    return min(times, key=times.get)


def _apply(cfg, knobs, system=None):
    """cfg with the knobs set; spme_grid_step picks the grid from the
    system's own candidates."""
    c = dataclasses.replace(cfg)
    for k, val in knobs.items():
        if k == "spme_grid_step":
            cands = grid_candidates(system, cfg)
            c.spme_grid = tuple(cands[min(int(val), len(cands) - 1)])
        elif k == "spme_grid":
            c.spme_grid = tuple(val)
        else:
            setattr(c, k, val)
    return c


def time_steps(system, cfg, steps=100, warmup=20, stream=None):
    """Seconds per step of MdState.step for this configuration: warmup steps,
    then steps steps between two synchronisations (host clock; the steps are
    captured graphs launched back to back, so the host clock sees the device
    time plus one synchronisation)."""
    st = md.MdState(system, cfg, stream=stream)
    try:
        st.step(0.002, warmup)
        st.sync()
        t0 = time.perf_counter()
        st.step(0.002, steps)
        st.sync()
        return (time.perf_counter() - t0) / steps
    finally:
        st.close()


def tune(system, cfg, steps=100, warmup=20, tie=0.02, cache=True, stream=None, log=None):
    """Chooses the knobs for this system (or its size class's cached choice).
    Returns {knob: value} and, with cache, stores it."""
    key = size_class(system, cfg)
    if cache:
        hit = lookup(key)
        if hit is not None:
            return dict(hit)
    cur = {"neighbor_skin": float(cfg.neighbor_skin), "prune_buffer": float(cfg.prune_buffer or 0.4),
           "ww_union_chunk": int(cfg.ww_union_chunk), "ww_split": int(cfg.ww_split),
           "pair_item_entries": int(cfg.pair_item_entries or 8),
           "spme_grid_step": 0}
    has_water = len(np.asarray(system.get("water_pos", np.zeros((0, 3, 3))))) > 0
    has_atoms = len(np.asarray(system.get("atom_pos", np.zeros((0, 3))))) > 0
    space = [("neighbor_skin", SKINS), ("prune_buffer", PRUNES if has_water else ()),
             ("ww_union_chunk", CHUNKS if has_water else ()),
             ("ww_split", SPLITS if has_water else ()),
             ("pair_item_entries", ITEMS if has_atoms else ()),
             ("spme_grid_step", tuple(range(len(grid_candidates(system, cfg)))))]
    measured = {}
    for knob, values in space:
        if not values:
            continue
        times = {}
        order = [cur[knob]] + [x for x in values if x != cur[knob]]
        for val in order:
            trial = dict(cur, **{knob: val})
            times[val] = time_steps(system, _apply(cfg, trial, system), steps, warmup, stream)
        cur[knob] = pick(times, order, tie)
        measured[knob] = {str(k): round(v * 1e3, 5) for k, v in times.items()}
        if log:
            log(f"{key} {knob}: {measured[knob]} -> {cur[knob]}")
    if cache:
        store = load_cache()
        store[key] = {"knobs": dict(cur), "ms_per_step": measured, "steps": steps,
                      "grid_chosen": list(_apply(cfg, cur, system).spme_grid)}
        save_cache(store)
    return cur


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def load_cache():
    """The user's cache (the classes tuned on this machine)."""
    return _load(cache_path())


def lookup(key):
    """The knobs of a size class: the user's cache first, then the shipped
    table; None when neither has it."""
    for store in (load_cache(), _load(SHIPPED)):
        if key in store:
            return store[key]["knobs"]
    return None


def save_cache(store):
    p = cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as f:
        json.dump(store, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


def apply_tuned(system, cfg, tune_missing=False, **kw):
    """cfg with the cached choice of its size class applied (tuned now with
    tune_missing, else the cfg unchanged when the class is not cached)."""
    hit = lookup(size_class(system, cfg))
    if hit is not None:
        return _apply(cfg, hit, system)
    if tune_missing:
        return _apply(cfg, tune(system, cfg, **kw), system)
    return cfg
