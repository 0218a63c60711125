"""Parity of the gpu_interface.rs drop-in (dyn_nb_*) with the oracle.

* the GPU-built flat pair list is bit-identical to the reference's
  brute-force lists + setup_pairs (src/neighbors.rs:102-281,
  src/non_bonded.rs:541-677) restated in exact float32 arithmetic;
* dyn_nb_forces matches the float64 evaluation of the same pair list with
  the reference CUDA kernel's conventions (src/cuda/cuda.cu:239-316) and with
  the CPU path's (src/non_bonded.rs:950-1057);
* results are bit-identical from call to call (64-bit fixed-point sums);
* with one molecule decoupled (alch_interaction pairs), dyn_nb_forces_alch
  matches the float64 evaluation of the alchemical pair kernel
  (src/cuda/cuda.cu:367-566) and of the CPU path, dH/dlambda included.
"""
import numpy as np
import pytest

from dynamics_b200 import gpu_interface as gi
from dynamics_b200 import synth
from oracle import pairs as opairs

from .systems import mixed, rel_rms, water_only

pytestmark = pytest.mark.gpu

CUTOFF = 10.0
SKIN = 4.0  # the reference default (src/config.rs:127)
ALPHA = synth.ewald_alpha(CUTOFF)
FORCE_RTOL = 1e-5   # per-atom force relative RMS vs float64
SCALAR_RTOL = 1e-5  # virial / energy relative error vs float64


def _build(sysd, lj_cutoff=0.0, cutoff=CUTOFF):
    na = len(sysd["atom_pos"])
    nw = len(sysd["water_pos"])
    fp = gi.ForcesPositsGpu(na, nw, cutoff, synth.ewald_alpha(cutoff), lj_cutoff)
    pn = gi.PerNeighborGpu.build(
        fp, sysd["atom_pos"], sysd["water_pos"][:, 0] if nw else None, sysd["atom_q"],
        sysd["atom_sigma"], sysd["atom_eps"], sysd["box_lo"], sysd["box_hi"], SKIN,
        excl=sysd.get("excl"), pair14=sysd.get("pair14"))
    return fp, pn


def _oracle_pairs(sysd, cutoff=CUTOFF):
    lists = opairs.build_all_neighbors(sysd, SKIN, cutoff)
    return opairs.setup_pairs(sysd, lists)


def _positions(sysd):
    pos_dyn, pw = opairs.site_positions(sysd)
    return pos_dyn, pw


def _check_pair_set(sysd, cutoff=CUTOFF):
    fp, pn = _build(sysd, cutoff=cutoff)
    got = pn.get_pairs()
    ref = _oracle_pairs(sysd, cutoff)
    assert pn.n_pairs == len(ref["tgt"])
    np.testing.assert_array_equal(got["tgt"], ref["tgt"])
    np.testing.assert_array_equal(got["src"], ref["src"])
    bt = np.where(ref["atype_tgt"] == 0, 0, ref["wtype_tgt"])
    bs = np.where(ref["atype_src"] == 0, 0, ref["wtype_src"])
    np.testing.assert_array_equal(got["body_tgt"], bt)
    np.testing.assert_array_equal(got["body_src"], bs)
    np.testing.assert_array_equal(got["flags"] & 1, ref["scale_14"])
    np.testing.assert_array_equal(got["flags"] & 8, ref["symmetric"] * 8)
    np.testing.assert_array_equal(got["sigma"], ref["sigma"])
    lj_eps = np.where(ref["calc_lj"] == 1, ref["eps"], 0).astype(np.float32)
    np.testing.assert_array_equal(got["eps"], lj_eps)
    qq = np.where(ref["calc_coulomb"] == 1, ref["q_tgt"] * ref["q_src"], 0).astype(np.float32)
    np.testing.assert_array_equal(got["qq"], qq)
    fp.close()


@pytest.mark.parametrize("make", [water_only, mixed])
def test_pair_set_bit_exact(gpu_lib, make):
    _check_pair_set(make())


def _c2_water_box():
    return synth.water_box(7800, 62.0, seed=2)


@pytest.mark.parametrize("make,cutoff", [(synth.config1, 10.0), (_c2_water_box, 9.0)], ids=["config1", "c2_size"])
def test_pair_set_bit_exact_baseline_sizes(gpu_lib, make, cutoff):
    """The reference's own system sizes.  The 512-water 24.8 A box breaks the
    reference's L > 2 (cutoff + skin) advice (src/lib.rs:560-561): the 14 A
    list radius exceeds half the box, so membership rests on the min-image
    rounding alone (0.89 M flat pairs).  A 62 A water box (7,800
    waters, 62 A, cutoff 9) has 14.8 M flat pairs."""
    _check_pair_set(make(), cutoff)


def test_pair_set_boundary_cases(gpu_lib):
    """Pairs at exactly the list radius and at half the box, where the
    reference's ties-away rounding and float32 order decide membership."""
    box = 30.0
    rl = CUTOFF + SKIN
    o = np.array([
        [1.0, 1.0, 1.0], [1.0 + rl, 1.0, 1.0],                 # exactly at the radius
        [5.0, 5.0, 5.0], [5.0 + np.nextafter(np.float32(rl), np.float32(0)), 5.0, 5.0],
        [20.0, 20.0, 20.0], [20.0, 20.0, 20.0 - 15.0],         # exactly half the box
        [0.0, 29.999998, 15.0], [0.0, 0.0, 15.0],              # across the face
    ], dtype=np.float32)
    quat = np.tile(np.array([1.0, 0, 0, 0]), (len(o), 1))
    h0, h1 = synth.water_geometry(o.astype(np.float64), quat)
    sysd = {
        "box_lo": np.zeros(3, np.float32), "box_hi": np.full(3, box, np.float32),
        "water_pos": np.stack([o, h0, h1], axis=1).astype(np.float32),
        "atom_pos": o[:3] + np.float32(0.7), "atom_q": np.array([1, -1, 0.5], np.float32),
        "atom_sigma": np.full(3, 3.0, np.float32), "atom_eps": np.full(3, 0.1, np.float32),
    }
    fp, pn = _build(sysd)
    got = pn.get_pairs()
    ref = _oracle_pairs(sysd)
    np.testing.assert_array_equal(got["tgt"], ref["tgt"])
    np.testing.assert_array_equal(got["src"], ref["src"])
    fp.close()


@pytest.mark.parametrize("make", [water_only, mixed])
@pytest.mark.parametrize("lj_cutoff", [0.0, CUTOFF])
def test_forces_match_float64(gpu_lib, make, lj_cutoff):
    sysd = make()
    fp, pn = _build(sysd, lj_cutoff)
    ref = _oracle_pairs(sysd)
    pos_dyn, pw = _positions(sysd)
    ext = (sysd["box_hi"] - sysd["box_lo"]).astype(np.float32)
    fd, fw, vir, en = gi.force_nonbonded_gpu(fp, pn, pos_dyn, pw, ext)
    f, e_ref, v_ref, _ = opairs.pair_forces(ref, pos_dyn, pw, ext, CUTOFF, ALPHA,
                                            lj_cutoff=lj_cutoff if lj_cutoff > 0 else None,
                                            gpu_semantics=lj_cutoff <= 0)
    rd, rw = opairs.accumulate_pair_forces(ref, f, len(pos_dyn), len(pw[1]))
    got = np.concatenate([fd.reshape(-1)] + [fw[k].reshape(-1) for k in (1, 2, 3, 4)])
    exp = np.concatenate([rd.reshape(-1)] + [rw[k].reshape(-1) for k in (1, 2, 3, 4)])
    assert rel_rms(got, exp) < FORCE_RTOL
    assert abs(vir - v_ref) <= SCALAR_RTOL * abs(v_ref)
    if abs(e_ref) > 0:
        assert abs(en - e_ref) <= SCALAR_RTOL * max(abs(e_ref), 1.0)
    fp.close()


def test_forces_bit_identical_across_calls(gpu_lib):
    sysd = mixed()
    fp, pn = _build(sysd)
    pos_dyn, pw = _positions(sysd)
    ext = (sysd["box_hi"] - sysd["box_lo"]).astype(np.float32)
    a = gi.force_nonbonded_gpu(fp, pn, pos_dyn, pw, ext)
    b = gi.force_nonbonded_gpu(fp, pn, pos_dyn, pw, ext)
    np.testing.assert_array_equal(a[0], b[0])
    for k in (1, 2, 3, 4):
        np.testing.assert_array_equal(a[1][k], b[1][k])
    assert a[2] == b[2] and a[3] == b[3]
    fp.close()


def test_set_pairs_matches_build(gpu_lib):
    sysd = mixed()
    ref = _oracle_pairs(sysd)
    na, nw = len(sysd["atom_pos"]), len(sysd["water_pos"])
    fp1, pn1 = _build(sysd)
    fp2 = gi.ForcesPositsGpu(na, nw, CUTOFF, ALPHA)
    pn2 = gi.PerNeighborGpu(fp2, ref)
    pos_dyn, pw = _positions(sysd)
    ext = (sysd["box_hi"] - sysd["box_lo"]).astype(np.float32)
    a = gi.force_nonbonded_gpu(fp1, pn1, pos_dyn, pw, ext)
    b = gi.force_nonbonded_gpu(fp2, pn2, pos_dyn, pw, ext)
    np.testing.assert_array_equal(a[0], b[0])
    assert a[2] == b[2]
    fp1.close()
    fp2.close()


ALCH_MOL = (5, 10)  # the second chain of systems.mixed


@pytest.mark.parametrize("lam", [0.0, 0.3, 0.75, 1.0])
@pytest.mark.parametrize("lj_cutoff", [0.0, CUTOFF])
def test_alchemical_forces_match_float64(gpu_lib, lam, lj_cutoff):
    sysd = mixed()
    fp, pn = _build(sysd, lj_cutoff)
    n_marked = pn.mark_alchemical(*ALCH_MOL)
    ref = opairs.setup_pairs(sysd, opairs.build_all_neighbors(sysd, SKIN, CUTOFF), alch_range=ALCH_MOL)
    assert n_marked == int(ref["alch"].sum()) > 0
    np.testing.assert_array_equal((pn.get_pairs()["flags"] & 16) != 0, ref["alch"] == 1)
    pos_dyn, pw = _positions(sysd)
    ext = (sysd["box_hi"] - sysd["box_lo"]).astype(np.float32)
    fd, fw, vir, en, dh = gi.force_nonbonded_gpu(fp, pn, pos_dyn, pw, ext, lambda_alch=lam)
    f, e_ref, v_ref, _, dh_ref = opairs.pair_forces(
        ref, pos_dyn, pw, ext, CUTOFF, ALPHA, lj_cutoff=lj_cutoff if lj_cutoff > 0 else None,
        gpu_semantics=lj_cutoff <= 0, lambda_alch=lam)
    rd, rw = opairs.accumulate_pair_forces(ref, f, len(pos_dyn), len(pw[1]))
    got = np.concatenate([fd.reshape(-1)] + [fw[k].reshape(-1) for k in (1, 2, 3, 4)])
    exp = np.concatenate([rd.reshape(-1)] + [rw[k].reshape(-1) for k in (1, 2, 3, 4)])
    assert rel_rms(got, exp) < FORCE_RTOL
    assert abs(vir - v_ref) <= SCALAR_RTOL * abs(v_ref)
    assert abs(en - e_ref) <= SCALAR_RTOL * max(abs(e_ref), 1.0)
    assert abs(dh - dh_ref) <= SCALAR_RTOL * max(abs(dh_ref), 1.0)
    fp.close()


def test_alchemical_flags_from_set_pairs(gpu_lib):
    """An alch column passed to set_pairs gives the same forces as marking
    the built list; clearing the marks restores the plain kernel."""
    sysd = mixed()
    ref = opairs.setup_pairs(sysd, opairs.build_all_neighbors(sysd, SKIN, CUTOFF), alch_range=ALCH_MOL)
    na, nw = len(sysd["atom_pos"]), len(sysd["water_pos"])
    fp1, pn1 = _build(sysd)
    pn1.mark_alchemical(*ALCH_MOL)
    fp2 = gi.ForcesPositsGpu(na, nw, CUTOFF, ALPHA)
    pn2 = gi.PerNeighborGpu(fp2, ref)
    pos_dyn, pw = _positions(sysd)
    ext = (sysd["box_hi"] - sysd["box_lo"]).astype(np.float32)
    a = gi.force_nonbonded_gpu(fp1, pn1, pos_dyn, pw, ext, lambda_alch=0.6)
    b = gi.force_nonbonded_gpu(fp2, pn2, pos_dyn, pw, ext, lambda_alch=0.6)
    np.testing.assert_array_equal(a[0], b[0])
    assert a[2] == b[2] and a[3] == b[3] and a[4] == b[4]
    assert pn1.mark_alchemical(0, 0) == 0
    plain = gi.force_nonbonded_gpu(fp1, pn1, pos_dyn, pw, ext)
    cleared = gi.force_nonbonded_gpu(fp1, pn1, pos_dyn, pw, ext, lambda_alch=0.6)
    np.testing.assert_array_equal(plain[0], cleared[0])
    assert cleared[4] == 0.0
    fp1.close()
    fp2.close()


def test_overrides_disable_terms(gpu_lib):
    sysd = mixed()
    fp, pn = _build(sysd)
    pos_dyn, pw = _positions(sysd)
    ext = (sysd["box_hi"] - sysd["box_lo"]).astype(np.float32)
    full = gi.force_nonbonded_gpu(fp, pn, pos_dyn, pw, ext)
    no_lj = gi.force_nonbonded_gpu(fp, pn, pos_dyn, pw, ext, overrides=2)
    no_c = gi.force_nonbonded_gpu(fp, pn, pos_dyn, pw, ext, overrides=1)
    both = gi.force_nonbonded_gpu(fp, pn, pos_dyn, pw, ext, overrides=3)
    assert np.all(both[0] == 0) and both[2] == 0.0
    np.testing.assert_allclose(no_lj[0] + no_c[0], full[0], rtol=0, atol=1e-6)
    fp.close()


def test_empty_pair_list(gpu_lib):
    """No installed pairs: every force, the virial and the energy are zero."""
    sysd = mixed()
    na, nw = len(sysd["atom_pos"]), len(sysd["water_pos"])
    fp = gi.ForcesPositsGpu(na, nw, CUTOFF, ALPHA)
    pn = gi.PerNeighborGpu(fp)
    pos_dyn, pw = _positions(sysd)
    ext = (sysd["box_hi"] - sysd["box_lo"]).astype(np.float32)
    fd, fw, vir, en, dh = gi.force_nonbonded_gpu(fp, pn, pos_dyn, pw, ext, lambda_alch=0.5)
    assert np.all(fd == 0) and all(np.all(fw[k] == 0) for k in (1, 2, 3, 4))
    assert vir == 0.0 and en == 0.0 and dh == 0.0
    assert pn.mark_alchemical(0, na) == 0
    fp.close()


def test_invalid_arguments_raise(gpu_lib):
    from dynamics_b200 import DynError
    with pytest.raises(DynError):
        gi.ForcesPositsGpu(1, 1, -1.0, 0.3)
    fp = gi.ForcesPositsGpu(2, 0, CUTOFF, ALPHA)
    bad = {"tgt": [0], "src": [5], "sigma": [3.0], "eps": [0.1], "q_tgt": [1.0], "q_src": [1.0],
           "body_tgt": [0], "body_src": [0], "scale_14": [0], "calc_lj": [1], "calc_coulomb": [1],
           "symmetric": [1]}
    with pytest.raises(DynError):
        gi.PerNeighborGpu(fp, bad)
    pn = gi.PerNeighborGpu(fp)
    with pytest.raises(DynError):
        pn.mark_alchemical(1, 3)   # beyond the two atoms
    with pytest.raises(DynError):
        gi.force_nonbonded_gpu(fp, pn, np.zeros((2, 3)), [np.zeros((0, 3))] * 4, [20.0] * 3,
                               lambda_alch=float("nan"))
    fp.close()
