"""Bonded forces and hydrogen constraints, float64 (oracle).

Restates apply_bonded_forces (src/bonded.rs:23-135) with the term forms of
src/bonded_forces.rs:
  bonds      U = k_b (r - r0)^2                     (:11-33)
  angles     U = k (theta - theta0)^2               (:37-81)
  dihedrals  U = sum k (1 + cos(n phi - phase))     (:84-178), phi the
             IUPAC/Amber dihedral; propers and impropers share the form.
Forces are the exact negative gradients (the reference's Blondel-Karplus
expressions evaluate the same gradient), and the virial uses the reference's
per-term relative-vector sums (src/bonded.rs:44-46,76-83,124-130).
System-dict keys: bonds (n,2) + bond_k, bond_r0; angles (n,3) + angle_k,
angle_theta0; dihedrals (n,4) + dihedral_k, dihedral_n, dihedral_phase (one
row per Fourier term; impropers are rows too).
"""
import numpy as np


def _mi(d, ext):
    return d - np.round(d / ext) * ext


def bonds(pos, idx, k, r0, ext):
    i, j = idx[:, 0], idx[:, 1]
    d = _mi(pos[j] - pos[i], ext)  # posit_1 - posit_0
    r = np.sqrt(np.sum(d * d, axis=1))
    dr = r - r0
    fmag = 2.0 * k * dr / np.maximum(r, 1e-8)
    f0 = d * fmag[:, None]  # force on atom 0
    e = k * dr * dr
    w = np.sum(d * f0, axis=1)
    return f0, -f0, e, w


def angles(pos, idx, k, theta0, ext):
    a, b, c = idx[:, 0], idx[:, 1], idx[:, 2]
    v01 = _mi(pos[a] - pos[b], ext)
    v21 = _mi(pos[c] - pos[b], ext)
    l01 = np.sqrt(np.sum(v01 * v01, axis=1))
    l21 = np.sqrt(np.sum(v21 * v21, axis=1))
    u01 = v01 / l01[:, None]
    u21 = v21 / l21[:, None]
    cos_t = np.clip(np.sum(u01 * u21, axis=1), -1.0, 1.0)
    theta = np.arccos(cos_t)
    sin_t = np.maximum(np.sqrt(1.0 - cos_t * cos_t), 1e-8)
    dth = theta - theta0
    de = 2.0 * k * dth
    g0 = (u01 * cos_t[:, None] - u21) / (l01 * sin_t)[:, None]
    g2 = (u21 * cos_t[:, None] - u01) / (l21 * sin_t)[:, None]
    f0 = -g0 * de[:, None]
    f2 = -g2 * de[:, None]
    f1 = -(f0 + f2)
    e = k * dth * dth
    w = np.sum(v01 * f0, axis=1) + np.sum(v21 * f2, axis=1)
    return f0, f1, f2, e, w


def dihedral_angle(p0, p1, p2, p3, ext):
    """IUPAC dihedral (trans = pi) and the bond vectors used."""
    b1 = _mi(p1 - p0, ext)
    b2 = _mi(p2 - p1, ext)
    b3 = _mi(p3 - p2, ext)
    n1 = np.cross(b1, b2)
    n2 = np.cross(b2, b3)
    b2n = np.sqrt(np.sum(b2 * b2, axis=1))
    x = np.sum(n1 * n2, axis=1)
    y = np.sum(np.cross(n1, n2) * b2, axis=1) / b2n
    return np.arctan2(y, x), b1, b2, b3, n1, n2


def dihedrals(pos, idx, k, n, phase, ext):
    p0, p1, p2, p3 = (pos[idx[:, m]] for m in range(4))
    phi, b1, b2, b3, n1, n2 = dihedral_angle(p0, p1, p2, p3, ext)
    e = k * (1.0 + np.cos(n * phi - phase))
    dv = -k * n * np.sin(n * phi - phase)  # dU/dphi
    n1sq = np.sum(n1 * n1, axis=1)
    n2sq = np.sum(n2 * n2, axis=1)
    b2sq = np.sum(b2 * b2, axis=1)
    b2n = np.sqrt(b2sq)
    # gradients of phi (Bekker; Blondel & Karplus 1996)
    g0 = -(b2n / n1sq)[:, None] * n1
    g3 = (b2n / n2sq)[:, None] * n2
    ta = np.sum(b1 * b2, axis=1) / b2sq
    tb = np.sum(b3 * b2, axis=1) / b2sq
    g1 = -g0 - ta[:, None] * g0 + tb[:, None] * g3
    g2 = -g3 - tb[:, None] * g3 + ta[:, None] * g0
    # the inner-atom terms follow the reference's arrangement
    # (src/bonded_forces.rs:161-175); tests check them by finite differences.
    f =[-(dv[:, None] * g) for g in (g0, g1, g2, g3)]
    w = (np.sum(-b1 * f[0], axis=1) + np.sum(b2 * f[2], axis=1)
         + np.sum((b2 + b3) * f[3], axis=1))
    return f, e, w


def bonded_forces(sysd, ext):
    pos = np.asarray(sysd["atom_pos"], dtype=np.float32).reshape(-1, 3).astype(np.float64)
    n = len(pos)
    out = np.zeros((n, 3))
    e_tot = 0.0
    w_tot = 0.0
    if "bonds" in sysd and len(sysd["bonds"]):
        idx = np.asarray(sysd["bonds"], dtype=np.int64).reshape(-1, 2)
        f0, f1, e, w = bonds(pos, idx, np.asarray(sysd["bond_k"], np.float64), np.asarray(sysd["bond_r0"], np.float64), ext)
        np.add.at(out, idx[:, 0], f0)
        np.add.at(out, idx[:, 1], f1)
        e_tot += float(np.sum(e)); w_tot += float(np.sum(w))
    if "angles" in sysd and len(sysd["angles"]):
        idx = np.asarray(sysd["angles"], dtype=np.int64).reshape(-1, 3)
        f0, f1, f2, e, w = angles(pos, idx, np.asarray(sysd["angle_k"], np.float64),
                                  np.asarray(sysd["angle_theta0"], np.float64), ext)
        np.add.at(out, idx[:, 0], f0)
        np.add.at(out, idx[:, 1], f1)
        np.add.at(out, idx[:, 2], f2)
        e_tot += float(np.sum(e)); w_tot += float(np.sum(w))
    if "dihedrals" in sysd and len(sysd["dihedrals"]):
        idx = np.asarray(sysd["dihedrals"], dtype=np.int64).reshape(-1, 4)
        f, e, w = dihedrals(pos, idx, np.asarray(sysd["dihedral_k"], np.float64),
                            np.asarray(sysd["dihedral_n"], np.float64),
                            np.asarray(sysd["dihedral_phase"], np.float64), ext)
        for m in range(4):
            np.add.at(out, idx[:, m], f[m])
        e_tot += float(np.sum(e)); w_tot += float(np.sum(w))
    return out, e_tot, w_tot


def rattle(pos, vel, mass, cons, inv_mass_sum):
    """rattle_hydrogens (src/bonded.rs:288-304), one sweep, FP64."""
    for c in range(len(cons)):
        i, j = cons[c]
        r = pos[j] - pos[i]
        v = vel[j] - vel[i]
        lam = np.dot(v, r) / (inv_mass_sum[c] * max(np.dot(r, r), 1e-8))
        corr = r * lam
        vel[i] += corr / mass[i]
        vel[j] -= corr / mass[j]
