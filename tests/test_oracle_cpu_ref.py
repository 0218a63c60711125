"""The timed CPU baseline computes what the float64 oracle computes.

oracle/cpu_ref is the C++17/OpenMP restatement of the reference CPU path
that bench.py times (its cpu_baseline and --impl reference arm).  One force
evaluation of it (O(N^2) list with the 4 A skin, flat-pair forces in float32
with float64 sums, bonded terms, SPME with the 1-4 vacuum correction,
src/non_bonded.rs:258-412,681-790, src/bonded.rs:23-135) is compared with
oracle.method.all_forces in the reference convention on the same
coordinates: the 512-water C1 box and a box of waters with chain molecules
(exclusions, 1-4 pairs, bonds, angles, dihedrals).  Tolerances are the
engine's own bars: per-site force relative RMS <= 1e-5, reciprocal energy
relative <= 1e-6.
"""
import numpy as np

from dynamics_b200 import synth
from oracle import cpu_ref, method

from .systems import mixed, rel_rms

FORCE_RTOL = 1e-5
E_RTOL = 1e-6


def _compare(sysd, cutoff, grid):
    got = cpu_ref.forces_once(sysd, cutoff, grid)
    ref = method.all_forces(sysd, {"cutoff": cutoff, "lj_cutoff": cutoff,
                                   "alpha": float(np.float32(synth.ewald_alpha(cutoff))),
                                   "grid": grid, "mode": "reference"})
    fa = np.concatenate([got["f_atoms"].reshape(-1), got["f_water"].reshape(-1)])
    fr = np.concatenate([ref["f_atoms"].reshape(-1), ref["f_water"].reshape(-1)])
    return rel_rms(fa, fr), got, ref


def test_cpu_ref_forces_config1():
    err, got, ref = _compare(synth.config1(), 10.0, (32, 32, 32))
    assert err < FORCE_RTOL, f"force rel-RMS {err:.3e}"
    assert abs(got["e_recip"] - ref["e_recip"]) <= E_RTOL * abs(ref["e_recip"]), (got["e_recip"], ref["e_recip"])
    assert abs(got["virial_pairs"] - ref["virial_short"]) <= 1e-5 * abs(ref["virial_short"])


def test_cpu_ref_forces_with_molecules():
    sysd = mixed()
    err, got, ref = _compare(sysd, 8.0, (32, 32, 32))
    assert err < FORCE_RTOL, f"force rel-RMS {err:.3e}"
    assert got["f_atoms"].shape == ref["f_atoms"].shape
    assert abs(got["e_recip"] - ref["e_recip"]) <= E_RTOL * abs(ref["e_recip"]), (got["e_recip"], ref["e_recip"])
