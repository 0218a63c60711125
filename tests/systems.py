"""Small seeded test systems shared by the parity tests."""
import numpy as np

from dynamics_b200 import synth


def water_only(n_side=7, spacing=3.1, seed=0):
    n = n_side ** 3
    return synth.water_box(n, n_side * spacing, seed=seed)


def mixed(n_side=7, spacing=3.1, n_mol=6, mol_len=5, seed=1):
    """Waters plus ``n_mol`` chain molecules of ``mol_len`` LJ+charge atoms.

    Each chain is a zig-zag with 1.5 A bonds; 1-2 and 1-3 pairs are
    exclusions, 1-4 pairs are scaled, every bond/angle/dihedral carries a
    harmonic/periodic term.  Waters within 2.6 A of an atom are removed.
    """
    rng = np.random.default_rng(seed)
    box = n_side * spacing
    atoms = []
    while len(atoms) < n_mol * mol_len:
        start = rng.uniform(2, box - 2, 3)
        dirn = rng.normal(size=3)
        dirn /= np.linalg.norm(dirn)
        perp = np.cross(dirn, rng.normal(size=3))
        perp /= np.linalg.norm(perp)
        chain = [start + dirn * 1.25 * k + perp * (0.45 if k % 2 else -0.45) for k in range(mol_len)]
        if atoms:
            d = np.array(chain)[:, None, :] - np.array(atoms)[None, :, :]
            d -= np.round(d / box) * box
            if np.min(np.linalg.norm(d, axis=2)) < 3.5:
                continue
        atoms.extend(chain)
    ap = np.array(atoms)
    na = len(ap)
    sites, _ = synth.lattice_sites(box, n_side ** 3)
    d = sites[:, None, :] - ap[None, :, :]
    d -= np.round(d / box) * box
    keep = np.min(np.linalg.norm(d, axis=2), axis=1) > 2.6
    wsys = synth.water_box(int(keep.sum()), box, seed=seed, sites=sites[keep])
    q = rng.normal(size=na) * 0.4
    q -= q.mean()
    excl, p14, bonds, angles, dih = [], [], [], [], []
    for m in range(n_mol):
        b = m * mol_len
        for k in range(mol_len - 1):
            excl.append((b + k, b + k + 1))
            bonds.append((b + k, b + k + 1))
        for k in range(mol_len - 2):
            excl.append((b + k, b + k + 2))
            angles.append((b + k, b + k + 1, b + k + 2))
        for k in range(mol_len - 3):
            p14.append((b + k, b + k + 3))
            dih.append((b + k, b + k + 1, b + k + 2, b + k + 3))
    bonds = np.array(bonds)
    r0 = np.linalg.norm(ap[bonds[:, 1]] - ap[bonds[:, 0]], axis=1)
    angles = np.array(angles)
    v1 = ap[angles[:, 0]] - ap[angles[:, 1]]
    v2 = ap[angles[:, 2]] - ap[angles[:, 1]]
    th0 = np.arccos(np.sum(v1 * v2, 1) / np.linalg.norm(v1, axis=1) / np.linalg.norm(v2, axis=1))
    wsys.update({
        "atom_pos": ap.astype(np.float32),
        "atom_vel": (rng.normal(size=(na, 3)) * 2.0).astype(np.float32),
        "atom_mass": np.full(na, 12.0, np.float32),
        "atom_q": (q * float(synth.CHARGE_UNIT_SCALER)).astype(np.float32),
        "atom_sigma": rng.uniform(2.6, 3.6, na).astype(np.float32),
        "atom_eps": rng.uniform(0.03, 0.15, na).astype(np.float32),
        "excl": np.array(excl, np.uint32), "pair14": np.array(p14, np.uint32),
        "bonds": bonds.astype(np.uint32), "bond_k": np.full(len(bonds), 300.0, np.float32),
        "bond_r0": r0.astype(np.float32),
        "angles": angles.astype(np.uint32), "angle_k": np.full(len(angles), 60.0, np.float32),
        "angle_theta0": th0.astype(np.float32),
        "dihedrals": np.array(dih, np.uint32), "dihedral_k": np.full(len(dih), 1.2, np.float32),
        "dihedral_n": np.full(len(dih), 3.0, np.float32), "dihedral_phase": np.zeros(len(dih), np.float32),
    })
    return wsys


def rel_rms(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))
