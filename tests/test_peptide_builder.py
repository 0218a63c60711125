"""Host-side synthetic peptide builder (no GPU): topology bookkeeping and
geometry of ff19SB peptides, and solvated systems with ions."""
import numpy as np

from dynamics_b200 import peptide, synth


def test_topology():
    p = peptide.build_peptide(["ALA", "GLY", "PRO", "TRP"], seed=1)
    n = len(p["atom_pos"])
    # a tree plus one ring bond in PRO and two in TRP
    assert len(p["bonds"]) == n - 1 + 3
    h = [i for i, nm in enumerate(p["names"]) if nm.startswith("H")]
    assert sorted(p["constraints"][:, 1].tolist()) == h   # every H constrained once
    ex = set(map(tuple, p["excl"].tolist()))
    for i, j in p["bonds"].tolist():
        assert (min(i, j), max(i, j)) in ex
    assert not ex & set(map(tuple, p["pair14"].tolist()))
    q = float(np.sum(p["atom_q"])) / float(synth.CHARGE_UNIT_SCALER)
    assert abs(q - p["net_charge"]) < 1e-4
    # bonded parameters found for every term
    assert np.all(p["bond_k"] > 0) and np.all(p["angle_k"] > 0)
    assert len(p["dihedrals"]) == len(p["dihedral_k"]) > 0


def test_geometry():
    rng = np.random.default_rng(3)
    p = peptide.build_peptide(peptide.random_sequence(20, rng), seed=3)
    x = p["atom_pos"].astype(np.float64)
    b = p["bonds"].astype(int)
    r = np.linalg.norm(x[b[:, 0]] - x[b[:, 1]], axis=1)
    assert np.max(np.abs(r - p["bond_r0"])) < 0.12
    from scipy.spatial import cKDTree
    skip = set(map(tuple, p["excl"].tolist())) | set(map(tuple, p["pair14"].tolist()))
    heavy = np.array([not nm.startswith("H") for nm in p["names"]])
    close = [(i, j) for i, j in cKDTree(x).query_pairs(2.2) if (min(i, j), max(i, j)) not in skip
             and heavy[i] and heavy[j]]
    assert not close


def test_solvated_system_is_neutral():
    sysd, seqs = peptide.solvated_system(30.0, 800, n_res=(10, 10), seed=5, nacl_molar=0.15)
    q = float(np.sum(sysd["atom_q"])) / float(synth.CHARGE_UNIT_SCALER)
    assert abs(q) < 1e-3
    n_pep = sum(len(peptide.build_peptide(s, seed=0)["atom_pos"]) for s in seqs)
    n_ions = len(sysd["atom_pos"]) - n_pep
    assert len(sysd["water_pos"]) == 800 - n_ions
    assert len(seqs) == 2 and all(len(s) == 10 for s in seqs)
