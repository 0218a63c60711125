"""The oracle's alchemical decoupling (soft-core LJ, scaled Coulomb, mixed
SPME on the staged schedule, src/alchemical.rs and src/non_bonded.rs):
dH/dlambda equals the finite difference of the potential energy, and the
forces are the energy's negative gradient."""
import numpy as np
import pytest

from dynamics_b200 import peptide, synth
from oracle import method


@pytest.fixture(scope="module")
def small():
    sysd, _ = peptide.solvated_system(24.8, 420, n_res=(2,), seed=5)
    n_pep = int(np.max(sysd["bonds"])) + 1  # the peptide's atoms come first; ions have no bonds
    return sysd, n_pep


def _params(n_pep, lam, mode="corrected"):
    return {"cutoff": 9.0, "lj_cutoff": 9.0, "alpha": synth.ewald_alpha(9.0), "grid": (24, 24, 24),
            "mode": mode, "alch_range": (0, n_pep), "alch_lambda": lam}


def test_schedule():
    assert method.decoupling_schedule(0.0) == (1.0, -2.0, 0.0, 0.0)
    assert method.decoupling_schedule(0.25) == (0.5, -2.0, 0.0, 0.0)
    assert method.decoupling_schedule(0.75) == (0.0, 0.0, 0.5, 2.0)
    assert method.decoupling_schedule(1.0) == (0.0, 0.0, 1.0, 2.0)


@pytest.mark.parametrize("lam", [0.3, 0.7])
def test_dhdl_is_energy_derivative(small, lam):
    sysd, n_pep = small
    h = 1e-4
    ep = method.all_forces(sysd, _params(n_pep, lam + h))["pe"]
    em = method.all_forces(sysd, _params(n_pep, lam - h))["pe"]
    dh = method.all_forces(sysd, _params(n_pep, lam))["dh_dl"]
    assert abs((ep - em) / (2 * h) - dh) <= 1e-5 * max(1.0, abs(dh)), ((ep - em) / (2 * h), dh)


@pytest.mark.parametrize("lam", [0.3, 0.7])
def test_alchemical_force_is_gradient(small, lam):
    sysd, n_pep = small
    r = method.all_forces(sysd, _params(n_pep, lam))
    a = 0  # an atom of the decoupled molecule
    h = 1e-4
    g = np.zeros(3)
    for k in range(3):
        d = {**sysd, "atom_pos": sysd["atom_pos"].astype(np.float64).copy()}
        d["atom_pos"][a, k] += h
        e1 = method.all_forces(d, _params(n_pep, lam))["pe"]
        d["atom_pos"][a, k] -= 2 * h
        e0 = method.all_forces(d, _params(n_pep, lam))["pe"]
        g[k] = (e1 - e0) / (2 * h)
    np.testing.assert_allclose(r["f_atoms"][a], -g, rtol=2e-3, atol=2e-3)


@pytest.mark.parametrize("lam", [0.0, 0.3, 0.75, 1.0])
def test_flat_pair_list_agrees_with_site_pairs(lam):
    """The flat-pair-list restatement (setup_pairs' alch_interaction column
    and the alchemical pair kernel's arithmetic) and the site-pair
    restatement (f_nonbonded_cpu over all site pairs) give the same forces,
    solute energy and dH/dlambda for one decoupled molecule."""
    from oracle import pairs as opairs
    from .systems import mixed
    cut = 10.0
    alpha = synth.ewald_alpha(cut)
    sysd = mixed()
    ref = opairs.setup_pairs(sysd, opairs.build_all_neighbors(sysd, 4.0, cut), alch_range=(5, 10))
    assert ref["alch"].sum() > 0
    pos_dyn, pw = opairs.site_positions(sysd)
    ext = (sysd["box_hi"] - sysd["box_lo"]).astype(np.float32)
    f, e, _, _, dh = opairs.pair_forces(ref, pos_dyn, pw, ext, cut, alpha, lj_cutoff=cut,
                                        lambda_alch=lam)
    fd, _ = opairs.accumulate_pair_forces(ref, f, len(pos_dyn), len(pw[1]))
    sr = method.short_range(sysd, cut, alpha, lj_cutoff=cut, alch=(5, 10, lam))
    assert abs(dh - sr["dh_dl"]) <= 1e-5 * max(abs(dh), 1.0)
    assert abs(e - sr["e_solute"]) <= 1e-5 * max(abs(e), 1.0)
    fs = sr["forces"][:len(pos_dyn)]
    assert np.sqrt(np.mean((fd - fs) ** 2)) <= 1e-5 * np.sqrt(np.mean(fs ** 2))
    if lam == 0.0:
        f0, e0, _, _ = opairs.pair_forces(ref, pos_dyn, pw, ext, cut, alpha, lj_cutoff=cut)
        np.testing.assert_allclose(f, f0, rtol=0, atol=1e-12)
        assert abs(e - e0) < 1e-10


def test_coincident_alchemical_pair():
    """A coincident alchemical pair: the CPU path keeps its soft-core contact
    energy and dH/dlambda with no force (src/non_bonded.rs:1002-1020), the
    GPU kernel skips it (r^2 < 1e-16, src/cuda/cuda.cu:448-450)."""
    from oracle import pairs as opairs
    pairs = {k: np.array(v) for k, v in {
        "tgt": [0], "src": [1], "sigma": [3.2], "eps": [0.15], "q_tgt": [0.4], "q_src": [-0.4],
        "atype_tgt": [0], "wtype_tgt": [0], "atype_src": [0], "wtype_src": [0], "scale_14": [0],
        "calc_lj": [1], "calc_coulomb": [1], "symmetric": [1], "alch": [1]}.items()}
    pos = np.array([[5.0, 5.0, 5.0], [5.0, 5.0, 5.0]], np.float32)
    pw = {s: np.zeros((0, 3)) for s in (1, 2, 3, 4)}
    lam = 0.8
    # the pair kernels take lambda as float32 (src/alchemical.rs:83)
    cs, dcs, ll, dll = method.decoupling_schedule(np.float32(lam))
    _, e_ref, dv = method.soft_core_lj(np.array([0.0]), np.array([3.2]), np.array([0.15]), ll)
    f, e, vir, _, dh = opairs.pair_forces(pairs, pos, pw, [20.0] * 3, 10.0, 0.3, lj_cutoff=10.0,
                                          lambda_alch=lam)
    assert np.all(f == 0.0) and vir == 0.0
    assert abs(e - float(e_ref[0])) < 1e-12 and e != 0.0
    assert abs(dh - float(dv[0]) * dll) < 1e-12
    f, e, vir, _, dh = opairs.pair_forces(pairs, pos, pw, [20.0] * 3, 10.0, 0.3, gpu_semantics=True,
                                          lambda_alch=lam)
    assert np.all(f == 0.0) and e == 0.0 and dh == 0.0
