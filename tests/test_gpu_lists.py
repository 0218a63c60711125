"""Completeness of the resident engine's neighbour lists.

The reference's lists hold every pair within cutoff + skin by construction
(O(N^2) scan, src/neighbors.rs:180-281).  The resident engine's lists are
cluster and molecule lists with a buffer, rebuilt when a molecule has moved
half the buffer (src/neighbors.rs:159-169); a pair missing from them would
only show as a small force error.  So the lists are read back
(dyn_sys_list_pairs) and every interacting pair inside the cutoff, found by
periodic k-d trees on the same coordinates, must be in them:

* at the list build, and at the last step before the next rebuild (where
  the molecules have moved the most since the build);
* on the c1 box (512 waters, 24.8 A, cutoff 10: the list radius exceeds
  half the box) at every step until the first rebuild, and on a box of
  waters with chain molecules (water-atom and atom-atom lists, exclusions,
  1-4 pairs); the 100k-atom c3 box is checked in test_gpu_precision.py.
"""
import numpy as np
import pytest

from dynamics_b200 import md, synth

from .coverage import covered_pairs, missing, needed_pairs
from .systems import mixed

pytestmark = pytest.mark.gpu


def check_lists(st, sysd, cutoff, state=None, covered=None):
    state = state if state is not None else st.state()
    covered = covered if covered is not None else covered_pairs(st, st.n_water, st.n_atoms)
    need = needed_pairs(state, sysd, cutoff)
    miss = missing(need, covered)
    for kind, (m, n) in enumerate(zip(miss, need)):
        assert len(m) == 0, f"list kind {kind}: {len(m)} of {len(n)} pairs inside the cutoff missing"
    return [len(n) for n in need]


def run_until_rebuild(st, sysd, cutoff, dt=0.002, max_steps=200, every_step=False):
    """Checks the lists at the build and at the last step before the next
    rebuild (with every_step, at every step in between too)."""
    counts = check_lists(st, sysd, cutoff)
    r0 = st.energies()["list_rebuilds"]
    prev = None
    for _ in range(max_steps):
        st.step(dt, 1)
        if st.energies()["list_rebuilds"] > r0:
            assert prev is not None, "rebuilt on the first step"
            check_lists(st, sysd, cutoff, *prev)
            return counts
        prev = (st.state(), covered_pairs(st, st.n_water, st.n_atoms))
        if every_step:
            check_lists(st, sysd, cutoff, *prev)
    raise AssertionError(f"no list rebuild within {max_steps} steps")


def test_lists_complete_config1(gpu_lib):
    sysd = synth.config1()
    cfg = md.MdConfig(coulomb_cutoff=10.0, lj_cutoff=10.0, spme_alpha=synth.ewald_alpha(10.0),
                      spme_grid=(32, 32, 32), integrator=md.LangevinMiddle(gamma=1.0), seed=3)
    st = md.MdState(sysd, cfg)
    counts = run_until_rebuild(st, sysd, 10.0, every_step=True)
    assert counts[0] > 30000  # 44.5 k water pairs with a site pair inside 10 A (measured)
    st.close()


def test_lists_complete_with_molecules(gpu_lib):
    sysd = mixed()
    cfg = md.MdConfig(coulomb_cutoff=8.0, lj_cutoff=8.0, spme_alpha=synth.ewald_alpha(8.0),
                      spme_grid=(32, 32, 32), integrator=md.LangevinMiddle(gamma=1.0), seed=4)
    st = md.MdState(sysd, cfg)
    counts = run_until_rebuild(st, sysd, 8.0, every_step=True)
    assert counts[1] > 0 and counts[2] > 0
    st.close()
