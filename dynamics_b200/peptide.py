"""Seeded random-sequence ff19SB peptides, solvated in OPC water with ions,
as synthetic inputs of the shapes the benchmarks name.

Residue templates, charges and bonded / LJ parameters come from the
reference's ff19SB files (amino19.lib, parm19.dat, frcmod.ff19SB, extracted
by data/make_ff19sb.py into data/ff19sb.json).  The chain is built from
ideal backbone internal coordinates (NeRF placement of N, CA, C), each
residue template superposed on its N, CA, C.  The chain is grown as a
self-avoiding random coil inside a sphere well inside the box (torsions from
the Ramachandran basins), so a chain far longer than the box (300 residues
in a 98 A cube) fits without touching its periodic image; an extended
meander of that length spans the whole box and drifts into its own
periodic image once it moves.  The termini are the internal templates (no
caps).  Ions: the reference's Joung-Cheatham OPC parameters
(src/lib.rs:1568-1658), placed on water sites that they replace.
"""
import json
import os

import numpy as np

from . import synth

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "ff19sb.json")
_FF = None

CHARGE_UNIT_SCALER = np.float32(18.2223)
STANDARD = ["ALA", "ARG", "ASN", "ASP", "CYS", "GLN", "GLU", "GLY", "HIE", "ILE", "LEU", "LYS", "MET",
            "PHE", "PRO", "SER", "THR", "TRP", "TYR", "VAL"]
# Joung-Cheatham ions for OPC (src/lib.rs:1577-1596): mass, charge (e), sigma, eps
IONS = {"Na+": (22.99, 1.0, 2.439, 0.1065), "Cl-": (35.45, -1.0, 4.478, 0.0073)}
SIGMA_FROM_RSTAR = 2.0 / 2.0 ** (1.0 / 6.0)


def ff():
    global _FF
    if _FF is None:
        _FF = json.load(open(_DATA))
    return _FF


def random_sequence(n, rng):
    return [STANDARD[i] for i in rng.integers(0, len(STANDARD), n)]


# ---------------------------------------------------------------------------
# geometry
# ---------------------------------------------------------------------------
def _place(a, b, c, bond, angle, torsion):
    """NeRF: position of d with |cd| = bond, angle(b, c, d) = angle and
    dihedral(a, b, c, d) = torsion (radians)."""
    bc = c - b
    bc /= np.linalg.norm(bc)
    n = np.cross(b - a, bc)
    n /= np.linalg.norm(n)
    m = np.cross(n, bc)
    d2 = np.array([-bond * np.cos(angle), bond * np.sin(angle) * np.cos(torsion),
                   bond * np.sin(angle) * np.sin(torsion)])
    return c + d2[0] * bc + d2[1] * m + d2[2] * n


def backbone(phi, psi, omega=None):
    """N, CA, C positions (n, 3, 3) from backbone torsions in degrees."""
    n = len(phi)
    omega = np.full(n, 180.0) if omega is None else omega
    r_nca, r_cac, r_cn = 1.458, 1.525, 1.329
    a_ncac, a_cacn, a_cnca = np.radians([111.2, 116.2, 121.7])
    out = np.zeros((n, 3, 3))
    out[0, 0] = [0.0, 0.0, 0.0]
    out[0, 1] = [r_nca, 0.0, 0.0]
    out[0, 2] = out[0, 1] + r_cac * np.array([-np.cos(a_ncac), np.sin(a_ncac), 0.0])
    for i in range(1, n):
        nn = _place(out[i - 1, 0], out[i - 1, 1], out[i - 1, 2], r_cn, a_cacn, np.radians(psi[i - 1]))
        ca = _place(out[i - 1, 1], out[i - 1, 2], nn, r_nca, a_cnca, np.radians(omega[i - 1]))
        cc = _place(out[i - 1, 2], nn, ca, r_cac, a_ncac, np.radians(phi[i]))
        out[i] = [nn, ca, cc]
    return out


def _kabsch(src, dst):
    """Rotation r and translation t with r @ src_i + t ~ dst_i."""
    cs, cd = src.mean(0), dst.mean(0)
    h = (src - cs).T @ (dst - cd)
    u, _, vt = np.linalg.svd(h)
    d = np.sign(np.linalg.det(vt.T @ u.T))
    r = vt.T @ np.diag([1.0, 1.0, d]) @ u.T
    return r, cd - r @ cs


def _place_v(a, b, c, bond, angle, torsion):
    """_place over candidates: a, b, c (m, 3); torsion (m,) radians."""
    bc = c - b
    bc /= np.linalg.norm(bc, axis=1, keepdims=True)
    n = np.cross(b - a, bc)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    m = np.cross(n, bc)
    return (c - bond * np.cos(angle) * bc + (bond * np.sin(angle) * np.cos(torsion))[:, None] * m
            + (bond * np.sin(angle) * np.sin(torsion))[:, None] * n)


def _grow(last, psi_last, phi, psi):
    """Backbone atoms of new residues after residue ``last`` (m, 3, 3) whose
    psi is psi_last (m,); phi, psi (m, r) in degrees.  Returns (m, r, 3, 3)."""
    r_nca, r_cac, r_cn = 1.458, 1.525, 1.329
    a_ncac, a_cacn, a_cnca = np.radians([111.2, 116.2, 121.7])
    m, r = phi.shape
    out = np.zeros((m, r, 3, 3))
    prev = last
    ps = np.radians(psi_last)
    om = np.full(m, np.pi)
    for k in range(r):
        nn = _place_v(prev[:, 0], prev[:, 1], prev[:, 2], r_cn, a_cacn, ps)
        ca = _place_v(prev[:, 1], prev[:, 2], nn, r_nca, a_cnca, om)
        cc = _place_v(prev[:, 2], nn, ca, r_cac, a_ncac, np.radians(phi[:, k]))
        out[:, k, 0], out[:, k, 1], out[:, k, 2] = nn, ca, cc
        prev = out[:, k]
        ps = np.radians(psi[:, k])
    return out


BETA = (-139.0, 135.0)


def _o_cb(bb, psi):
    """Carbonyl O and a CB of every residue of backbones bb (..., r, 3, 3)
    from ideal geometry (O anti to the next N; L-configuration CB)."""
    sh = bb.shape
    f = bb.reshape(-1, 3, 3)
    ps = np.radians(np.broadcast_to(psi, sh[:-2]).reshape(-1))
    o = _place_v(f[:, 0], f[:, 1], f[:, 2], 1.229, np.radians(120.5), ps + np.pi)
    cb = _place_v(f[:, 2], f[:, 0], f[:, 1], 1.53, np.radians(110.5), np.full(len(f), np.radians(-122.5)))
    return o.reshape(sh[:-2] + (3,)), cb.reshape(sh[:-2] + (3,))


# (phi, psi) basin centres and weights for the growth: beta, polyproline
# II, right- and left-handed helix
BASINS = np.array([[-120.0, 130.0], [-70.0, 145.0], [-63.0, -42.0], [57.0, 47.0]])
WEIGHTS = np.array([0.35, 0.30, 0.30, 0.05])


def coil_backbone(n_res, radius, seed=0, pro=(), gly=(), n_try=48, clear=3.0):
    """N, CA, C of a self-avoiding chain grown residue by residue inside a
    sphere of ``radius`` (on CA), each residue's (phi, psi) drawn from the
    Ramachandran basins (proline phi fixed at -65, glycine may also take the
    left-handed basin more often).  A candidate must keep its heavy backbone
    atoms (N, CA, C, CB and the previous residue's O) ``clear`` of every
    earlier residue but its neighbour; with no valid candidate the last
    residues are regrown."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    pro, gly = set(pro), set(gly)
    phi = np.full(n_res, -120.0)
    psi = np.full(n_res, 130.0)
    bb = np.zeros((n_res, 3, 3))
    bb[0] = backbone(phi[:1], psi[:1])[0]
    bb[0] -= bb[0, 1]
    _, cb0 = _o_cb(bb[:1], psi[:1])
    heavy = [np.concatenate([bb[0], cb0])]   # per residue: N, CA, C, CB (+ O once known)
    i, fails = 1, 0
    while i < n_res:
        w = WEIGHTS.copy()
        if i in gly:
            w[3] = 0.25
        w /= w.sum()
        pick = rng.choice(len(BASINS), n_try, p=w)
        ph = BASINS[pick, 0] + rng.normal(0, 12.0, n_try)
        if i in pro:
            ph[:] = -65.0
        # psi of residue i-1 places residue i
        ps_prev = BASINS[rng.choice(len(BASINS), n_try, p=WEIGHTS), 1] + rng.normal(0, 12.0, n_try)
        cand = _grow(np.repeat(bb[i - 1][None], n_try, 0), ps_prev, ph[:, None], np.zeros((n_try, 1)))[:, 0]
        o_prev, _ = _o_cb(bb[i - 1][None].repeat(n_try, 0), ps_prev)
        _, cb_new = _o_cb(cand, np.zeros(n_try))
        pts = np.concatenate([cand, cb_new[:, None], o_prev[:, None]], axis=1)  # (t, 5, 3)
        ok = np.linalg.norm(cand[:, 1], axis=1) < radius
        if i >= 3:
            tree = cKDTree(np.concatenate(heavy[:i - 1]))
            d, _ = tree.query(pts.reshape(-1, 3))
            ok &= d.reshape(n_try, -1).min(axis=1) >= clear
        if not ok.any():
            fails += 1
            if fails > 4000:
                raise RuntimeError("coil growth failed; use a larger radius")
            back = min(i - 1, 1 + fails // 8 % 4)
            i -= back
            heavy = heavy[:i]
            heavy[-1] = heavy[-1][:4]
            continue
        good = np.nonzero(ok)[0]
        rr = np.linalg.norm(cand[good, 1], axis=1)
        t = good[np.argmin(rr)] if rr.min() > 0.8 * radius else good[rng.integers(len(good))]
        phi[i], psi[i - 1] = ph[t], ps_prev[t]
        bb[i] = cand[t]
        heavy = heavy[:i]
        heavy[-1] = np.concatenate([heavy[-1][:4], o_prev[t][None]])
        heavy.append(np.concatenate([bb[i], cb_new[t][None]]))
        i += 1
    return bb, phi, psi


BACKBONE = {"N", "H", "CA", "HA", "HA2", "HA3", "C", "O"}


def _fix_peptide_planes(pos, names, res_of, n_res):
    """Puts each carbonyl O and amide H in its peptide plane: the template
    superposed on N, CA, C carries the template's psi and phi for them."""
    idx = {}
    for i, (nm, r) in enumerate(zip(names, res_of)):
        idx[(r, nm)] = i
    for r in range(n_res):
        c, ca = idx[(r, "C")], idx[(r, "CA")]
        if r + 1 < n_res and (r, "O") in idx:
            nn = idx[(r + 1, "N")]
            u = pos[ca] - pos[c]
            w = pos[nn] - pos[c]
            d = -(u / np.linalg.norm(u) + w / np.linalg.norm(w))
            pos[idx[(r, "O")]] = pos[c] + 1.229 * d / np.linalg.norm(d)
        if r > 0 and (r, "H") in idx:
            nn = idx[(r, "N")]
            u = pos[idx[(r - 1, "C")]] - pos[nn]
            w = pos[ca] - pos[nn]
            d = -(u / np.linalg.norm(u) + w / np.linalg.norm(w))
            pos[idx[(r, "H")]] = pos[nn] + 1.01 * d / np.linalg.norm(d)


def _side(nbr, a, b):
    """Atoms on b's side of the bond a-b (None if the bond is in a ring)."""
    seen, stack = {b}, [b]
    while stack:
        x = stack.pop()
        for y in nbr[x]:
            if x == b and y == a:
                continue
            if y == a:
                return None
            if y not in seen:
                seen.add(y)
                stack.append(y)
    return seen - {b}


def _rotate(p, axis_a, axis_b, ang):
    k = axis_b - axis_a
    k = k / np.linalg.norm(k)
    v = p - axis_b
    c, s = np.cos(ang), np.sin(ang)
    return axis_b + v * c + np.cross(k, v) * s + np.outer(v @ k, k) * (1.0 - c)


def _relieve_clashes(pos, names, res_of, nbr, seq, steps=12):
    """Turns side chains about their rotatable heavy-atom bonds, outward
    from CA, to the rotamer (30-degree grid) farthest from every atom that
    is more than three bonds away."""
    from scipy.spatial import cKDTree
    n = len(names)
    heavy = np.array([not nm.startswith("H") for nm in names])
    # atoms within three bonds of each atom (not clashes)
    near = []
    for i in range(n):
        s1 = nbr[i]
        s2 = set().union(*[nbr[j] for j in s1]) if s1 else set()
        s3 = set().union(*[nbr[j] for j in s2]) if s2 else set()
        near.append(s1 | s2 | s3 | {i})
    for r, rn in enumerate(seq):
        if rn in ("GLY", "ALA", "PRO"):
            continue
        atoms = np.nonzero(res_of == r)[0]
        byname = {names[i]: i for i in atoms}
        if "CA" not in byname or "CB" not in byname:
            continue
        # rotatable bonds outward from CA, breadth first over heavy atoms
        order, frontier, seen = [], [(byname["CA"], byname["CB"])], {byname["CA"], byname["CB"]}
        while frontier:
            a, b = frontier.pop(0)
            order.append((a, b))
            for c in sorted(nbr[b]):
                if c not in seen and heavy[c] and res_of[c] == r and names[c] not in BACKBONE:
                    seen.add(c)
                    frontier.append((b, c))
        for a, b in order:
            moving = _side(nbr, a, b)
            if not moving or sum(heavy[list(moving)]) < 1:
                continue
            mv = np.array(sorted(moving))
            others = np.setdiff1d(np.arange(n), np.concatenate([mv, [a, b]]))
            tree = cKDTree(pos[others])
            best, best_d = 0.0, -1.0
            for k in range(steps):
                ang = 2.0 * np.pi * k / steps
                pm = _rotate(pos[mv], pos[a], pos[b], ang)
                d, j = tree.query(pm, k=8, distance_upper_bound=4.0)
                dmin = 4.0
                for row, (dd, jj) in enumerate(zip(d, j)):
                    for x, y in zip(dd, jj):
                        if np.isfinite(x) and others[y] not in near[mv[row]]:
                            dmin = min(dmin, x)
                            break
                if dmin > best_d + 1e-6:
                    best, best_d = ang, dmin
            pos[mv] = _rotate(pos[mv], pos[a], pos[b], best)
    return pos


def relax(pos, bonds, r0, angles, theta0, skip, is_h, n_iter=600):
    """Removes close contacts by steepest descent on harmonic bonds and
    angles plus a soft repulsion between atoms closer than 3.0 A (heavy
    pairs), 2.5 A (heavy-H) or 2.0 A (H-H) that are not 1-2, 1-3 or 1-4
    partners.  A geometric clean-up of generated coordinates only."""
    from scipy.spatial import cKDTree
    x = pos.astype(np.float64).copy()
    is_h = np.asarray(is_h)
    step = 0.002
    prev_e = np.inf
    for it in range(n_iter):
        g = np.zeros_like(x)
        d = x[bonds[:, 1]] - x[bonds[:, 0]]
        r = np.linalg.norm(d, axis=1)
        e = np.sum(300.0 * (r - r0) ** 2)
        f = (600.0 * (r - r0) / np.maximum(r, 1e-6))[:, None] * d
        np.add.at(g, bonds[:, 1], f)
        np.add.at(g, bonds[:, 0], -f)
        a, b, c = angles[:, 0], angles[:, 1], angles[:, 2]
        u, v = x[a] - x[b], x[c] - x[b]
        lu, lv = np.linalg.norm(u, axis=1), np.linalg.norm(v, axis=1)
        ct = np.clip(np.sum(u * v, 1) / (lu * lv), -0.999999, 0.999999)
        th = np.arccos(ct)
        e += np.sum(60.0 * (th - theta0) ** 2)
        dth = -120.0 * (th - theta0) / np.sqrt(1.0 - ct * ct)
        ga = dth[:, None] * (v / (lu * lv)[:, None] - (ct / lu ** 2)[:, None] * u)
        gc = dth[:, None] * (u / (lu * lv)[:, None] - (ct / lv ** 2)[:, None] * v)
        np.add.at(g, a, ga)
        np.add.at(g, c, gc)
        np.add.at(g, b, -ga - gc)
        pr = cKDTree(x).query_pairs(3.0, output_type="ndarray")
        if len(pr):
            keep = np.array([(min(i, j), max(i, j)) not in skip for i, j in pr])
            pr = pr[keep]
        if len(pr):
            i, j = pr[:, 0], pr[:, 1]
            nh = is_h[i].astype(int) + is_h[j].astype(int)
            d0 = np.where(nh == 0, 3.0, np.where(nh == 1, 2.5, 2.0))
            dd = x[j] - x[i]
            rr = np.linalg.norm(dd, axis=1)
            over = np.maximum(0.0, d0 - rr)
            e += np.sum(100.0 * over ** 2)
            fr = (200.0 * over / np.maximum(rr, 1e-6))[:, None] * dd
            np.add.at(g, i, fr)
            np.add.at(g, j, -fr)
            if over.max() < 0.05 and it > 50:
                break
        step = step * 1.1 if e < prev_e else step * 0.5
        prev_e = e
        gn = np.linalg.norm(g, axis=1).max()
        x -= g * min(step, 0.05 / max(gn, 1e-12))
    return x


# ---------------------------------------------------------------------------
# topology and parameters
# ---------------------------------------------------------------------------
def _key(ty):
    ty = list(ty)
    return "-".join(ty) if ty <= ty[::-1] else "-".join(ty[::-1])


class _Params:
    def __init__(self):
        p = ff()["params"]
        self.mass = p["mass"]
        self.nonb = p["nonb"]
        self.bond = {_key(e[0]): (e[1], e[2]) for e in p["bond"]}
        self.angle = {_key(e[0]): (e[1], e[2]) for e in p["angle"]}
        self.dihe = {}
        for e in p["dihe"]:
            self.dihe.setdefault(_key(e[0]), []).append(e[1:])
        self.impr = [(e[0], e[1:]) for e in p["impr"]]

    def dihedral(self, ty):
        for k in (_key(ty), _key(["X", ty[1], ty[2], "X"])):
            if k in self.dihe:
                # (k, n, phase) per term: pk / idivf, |pn|, phase in radians
                return [(pk / idiv, abs(pn), np.radians(ph)) for idiv, pk, ph, pn in self.dihe[k]]
        return []

    def improper(self, t1, t2, t3, t4):
        best, score = None, -1
        for ty, par in self.impr:
            if ty[2] != t3:
                continue
            ok, s = True, 0
            for want, have in ((ty[0], t1), (ty[1], t2), (ty[3], t4)):
                if want == "X":
                    continue
                if want != have:
                    ok = False
                    break
                s += 1
            if ok and s > score:
                best, score = par, s
        return best, score


def build_peptide(seq, seed=0):
    """Atoms and bonded topology of a peptide of residue names ``seq``.

    Returns a dict with atom_pos (n, 3) centred at the origin, atom_mass,
    atom_q (scaled by 18.2223), atom_sigma, atom_eps, bonds + bond_k,
    bond_r0, angles + angle_k, angle_theta0, dihedrals (one row per term,
    propers and impropers) + dihedral_k / _n / _phase, excl (1-2, 1-3),
    pair14, constraints (bonds to H) + constraint_r0, net_charge (e)."""
    res_t = ff()["residues"]
    n_res = len(seq)
    radius = max(8.0, 2.2 * n_res ** (1.0 / 3.0) * 3.8 * 0.5 + 6.0)
    bb, _, _ = coil_backbone(n_res, radius, seed=seed, pro=[i for i, r in enumerate(seq) if r == "PRO"],
                             gly=[i for i, r in enumerate(seq) if r == "GLY"])
    # principal axes of the backbone along x, y, z (smallest box)
    c0 = bb.reshape(-1, 3).mean(0)
    _, _, vt = np.linalg.svd(bb.reshape(-1, 3) - c0, full_matrices=False)
    bb = (bb - c0) @ vt.T
    names, types, charges, pos, res_of = [], [], [], [], []
    bonds = []
    prev_tail = None
    for r, rn in enumerate(seq):
        t = res_t[rn]
        an = [a["name"] for a in t["atoms"]]
        idx = [an.index(x) for x in ("N", "CA", "C")]
        tp = np.asarray(t["pos"])
        rot, tr = _kabsch(tp[idx], bb[r])
        p = tp @ rot.T + tr
        base = len(names)
        names += an
        types += [a["type"] for a in t["atoms"]]
        charges += [a["charge"] for a in t["atoms"]]
        pos.append(p)
        res_of += [r] * len(an)
        bonds += [(base + i, base + j) for i, j in t["bonds"]]
        head, tail = base + t["connect"][0], base + t["connect"][1]
        if prev_tail is not None:
            bonds.append((prev_tail, head))
        prev_tail = tail
    pos = np.concatenate(pos)
    n = len(names)
    prm = _Params()
    nbr = [set() for _ in range(n)]
    for i, j in bonds:
        nbr[i].add(j)
        nbr[j].add(i)
    _fix_peptide_planes(pos, names, np.array(res_of), n_res)
    pos = _relieve_clashes(pos, names, np.array(res_of), nbr, seq)
    # bonds
    b_k, b_r0 = [], []
    for i, j in bonds:
        k, r0 = prm.bond[_key([types[i], types[j]])]
        b_k.append(k)
        b_r0.append(r0)
    # angles
    angles, a_k, a_t0 = [], [], []
    for j in range(n):
        nb = sorted(nbr[j])
        for x in range(len(nb)):
            for y in range(x + 1, len(nb)):
                i, k = nb[x], nb[y]
                kk, t0 = prm.angle[_key([types[i], types[j], types[k]])]
                angles.append((i, j, k))
                a_k.append(kk)
                a_t0.append(np.radians(t0))
    # proper dihedrals
    dih, d_k, d_n, d_ph = [], [], [], []
    pair14 = set()
    for j, k in bonds:
        for i in sorted(nbr[j] - {k}):
            for l in sorted(nbr[k] - {j}):
                if i == l:
                    continue
                for kk, nn, ph in prm.dihedral([types[i], types[j], types[k], types[l]]):
                    dih.append((i, j, k, l))
                    d_k.append(kk)
                    d_n.append(nn)
                    d_ph.append(ph)
                pair14.add((min(i, l), max(i, l)))
    # impropers: trigonal centres, central atom third (Amber convention)
    for k in range(n):
        if len(nbr[k]) != 3:
            continue
        nb = sorted(nbr[k])
        best = None
        for a, b_, c in ((nb[0], nb[1], nb[2]), (nb[0], nb[2], nb[1]), (nb[1], nb[2], nb[0])):
            for i, j in ((a, b_), (b_, a)):
                par, s = prm.improper(types[i], types[j], types[k], types[c])
                if par is not None and (best is None or s > best[0]):
                    best = (s, (i, j, k, c), par)
        if best is not None:
            pk, ph, pn = best[2]
            dih.append(best[1])
            d_k.append(pk)
            d_n.append(abs(pn))
            d_ph.append(np.radians(ph))
    # exclusions (1-2, 1-3) and 1-4 pairs
    excl = set()
    for i, j in bonds:
        excl.add((min(i, j), max(i, j)))
    for i, j, k in angles:
        excl.add((min(i, k), max(i, k)))
    pair14 = sorted(pair14 - excl)
    # constraints: bonds to hydrogen
    is_h = np.array([nm.startswith("H") for nm in names])
    cons, c_r0 = [], []
    for (i, j), r0 in zip(bonds, b_r0):
        if is_h[i] != is_h[j]:
            cons.append((j, i) if is_h[i] else (i, j))   # (heavy, H)
            c_r0.append(r0)
    pos = relax(pos, np.array(bonds), np.array(b_r0), np.array(angles).reshape(-1, 3), np.array(a_t0),
                excl | set(pair14), [nm.startswith("H") for nm in names])
    mass = np.array([prm.mass[t] for t in types], np.float32)
    rstar = np.array([prm.nonb[t][0] for t in types])
    eps = np.array([prm.nonb[t][1] for t in types], np.float32)
    q = np.array(charges, np.float64)
    pos = pos - pos.mean(0)
    return {
        "atom_pos": pos.astype(np.float32), "atom_mass": mass,
        "atom_q": (q.astype(np.float32) * CHARGE_UNIT_SCALER).astype(np.float32),
        "atom_sigma": (rstar * SIGMA_FROM_RSTAR).astype(np.float32), "atom_eps": eps,
        "bonds": np.array(bonds, np.uint32), "bond_k": np.array(b_k, np.float32),
        "bond_r0": np.array(b_r0, np.float32),
        "angles": np.array(angles, np.uint32).reshape(-1, 3), "angle_k": np.array(a_k, np.float32),
        "angle_theta0": np.array(a_t0, np.float32),
        "dihedrals": np.array(dih, np.uint32).reshape(-1, 4), "dihedral_k": np.array(d_k, np.float32),
        "dihedral_n": np.array(d_n, np.float32), "dihedral_phase": np.array(d_ph, np.float32),
        "excl": np.array(sorted(excl), np.uint32).reshape(-1, 2),
        "pair14": np.array(pair14, np.uint32).reshape(-1, 2),
        "constraints": np.array(cons, np.uint32).reshape(-1, 2),
        "constraint_r0": np.array(c_r0, np.float32),
        "names": names, "types": types, "residue": np.array(res_of),
        "net_charge": float(np.round(q.sum())),
    }


def _merge(parts):
    """Concatenates peptide dicts, offsetting their indices."""
    out = {}
    off = 0
    idx_keys = ("bonds", "angles", "dihedrals", "excl", "pair14", "constraints")
    for p in parts:
        n = len(p["atom_pos"])
        for k, v in p.items():
            if k in ("names", "types", "residue", "net_charge"):
                continue
            v = np.asarray(v)
            if k in idx_keys:
                v = v.astype(np.int64) + off
            out.setdefault(k, []).append(v)
        off += n
    res = {k: np.concatenate(v) for k, v in out.items()}
    for k in idx_keys:
        res[k] = res[k].astype(np.uint32)
    return res


def solvated_system(box, n_water, n_res=(), seed=0, nacl_molar=0.0, temperature=300.0):
    """Peptides of the given residue counts (random ff19SB sequences), OPC
    water filling the rest of a ``box`` cube, counter-ions to neutralise and
    NaCl at ``nacl_molar``.  Waters and ions sit on a jittered lattice; ions
    replace waters (src/lib.rs:1568-1658), so the water count ends up
    ``n_water`` minus the ions.  Returns an engine system dict (with
    constraints on bonds to hydrogen) and the sequences."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    peps, seqs = [], []
    placed = np.zeros((0, 3))
    for k, nr in enumerate(n_res):
        seq = random_sequence(int(nr), rng)
        p = build_peptide(seq, seed=seed * 100 + k)
        pos = p["atom_pos"].astype(np.float64)
        ok = False
        for _ in range(200):
            # first peptide at the centre; others anywhere clear of the rest
            c = np.full(3, box / 2.0) if k == 0 else rng.uniform(0.0, box, 3)
            trial = pos + c
            if len(placed) == 0:
                ok = True
                break
            t = cKDTree(np.mod(placed, box), boxsize=box)
            d, _ = t.query(np.mod(trial, box))
            if d.min() > 4.0:
                ok = True
                break
        if not ok:
            raise ValueError(f"no room for peptide {k} in a {box:.1f} A box")
        p["atom_pos"] = trial.astype(np.float32)
        placed = np.concatenate([placed, trial])
        peps.append(p)
        seqs.append(seq)
    solute = _merge(peps) if peps else None
    net = sum(p["net_charge"] for p in peps)
    vol = box ** 3
    n_pairs = int(round(nacl_molar * 6.02214076e-4 * vol))
    n_na = n_pairs + (int(round(-net)) if net < 0 else 0)
    n_cl = n_pairs + (int(round(net)) if net > 0 else 0)
    # lattice sites clear of the solute, then n_water of them for water
    excl_r = 2.6
    free_frac = 1.0
    sites = None
    for _ in range(6):
        need = int(np.ceil(n_water / free_frac * 1.02))
        sites, _ = synth.lattice_sites(box, need)
        if solute is not None:
            t = cKDTree(np.mod(solute["atom_pos"].astype(np.float64), box), boxsize=box)
            d, _ = t.query(np.mod(sites, box))
            keep = d > excl_r
        else:
            keep = np.ones(len(sites), bool)
        if keep.sum() >= n_water:
            break
        free_frac = max(0.05, keep.mean() * 0.95)
    sites = sites[keep]
    sites = sites[np.sort(rng.choice(len(sites), n_water, replace=False))]
    o = np.mod(sites + rng.uniform(-0.05, 0.05, sites.shape), box)
    # ions replace waters spread through the box
    n_ion = n_na + n_cl
    ion_idx = np.zeros(0, int)
    if n_ion:
        stride = max(1, n_water // n_ion)
        ion_idx = (np.arange(n_ion) * stride + stride // 2) % n_water
    ion_pos = o[ion_idx]
    o = np.delete(o, ion_idx, axis=0)
    quat = synth.orient_waters(o, box, rng, solute=None if solute is None else solute["atom_pos"])
    h0, h1 = synth.water_geometry(o, quat)
    wpos = np.stack([o, h0, h1], axis=1)
    wvel = synth.rigid_mb_velocities(wpos, temperature, rng)
    # atoms: peptides then ions
    kinds = ["Na+"] * n_na + ["Cl-"] * n_cl
    ion_mass = np.array([IONS[k][0] for k in kinds], np.float32)
    ion_q = np.array([IONS[k][1] for k in kinds], np.float32) * CHARGE_UNIT_SCALER
    ion_sig = np.array([IONS[k][2] for k in kinds], np.float32)
    ion_eps = np.array([IONS[k][3] for k in kinds], np.float32)
    if solute is None:
        solute = {k: np.zeros((0, 3) if k == "atom_pos" else 0, np.float32)
                  for k in ("atom_pos", "atom_mass", "atom_q", "atom_sigma", "atom_eps")}
    ap = np.concatenate([solute["atom_pos"], ion_pos.astype(np.float32)]).astype(np.float32)
    am = np.concatenate([solute["atom_mass"], ion_mass]).astype(np.float32)
    kt = float(synth.KB_NATIVE) * temperature
    av = (rng.normal(size=ap.shape) * np.sqrt(kt / np.maximum(am, 1e-6))[:, None])
    sysd = {
        "box_lo": np.zeros(3, np.float32), "box_hi": np.full(3, box, np.float32),
        "water_pos": wpos.astype(np.float32), "water_vel": wvel,
        "atom_pos": ap, "atom_vel": av, "atom_mass": am,
        "atom_q": np.concatenate([solute["atom_q"], ion_q]).astype(np.float32),
        "atom_sigma": np.concatenate([solute["atom_sigma"], ion_sig]).astype(np.float32),
        "atom_eps": np.concatenate([solute["atom_eps"], ion_eps]).astype(np.float32),
    }
    for k in ("bonds", "bond_k", "bond_r0", "angles", "angle_k", "angle_theta0", "dihedrals", "dihedral_k",
              "dihedral_n", "dihedral_phase", "excl", "pair14", "constraints", "constraint_r0"):
        if peps:
            sysd[k] = solute[k]
    n_cons = len(sysd.get("constraints", ()))
    dof = 6 * len(wpos) + 3 * len(ap) - n_cons - 3
    synth.remove_com_and_scale(sysd, temperature, dof)
    sysd["water_vel"] = sysd["water_vel"].astype(np.float32)
    sysd["atom_vel"] = sysd["atom_vel"].astype(np.float32)
    return sysd, seqs


def batch_member(n_water, n_peptides, seed=0, n_res=10, density=0.0334, spacing=1.0):
    """One member of the batched / served workloads: ``n_peptides`` random
    ``n_res``-residue peptides with counter-ions in a box of ``n_water`` OPC
    waters at ``density`` per cubic angstrom, and an FFT-friendly SPME grid
    of about ``spacing`` A.  If the peptides do not fit clear of each other
    (small boxes), other placements are tried, then one peptide fewer.
    Returns (system, grid, peptides placed)."""
    box = float((n_water / density) ** (1.0 / 3.0))
    k = synth.fft_size(int(np.ceil(box / spacing)))
    for n_pep in range(int(n_peptides), -1, -1):
        for attempt in range(4):
            try:
                sysd, _ = solvated_system(box, int(n_water), n_res=(n_res,) * n_pep,
                                          seed=seed * 16 + attempt)
                return sysd, (k, k, k), n_pep
            except ValueError:
                continue
    raise ValueError("batch member could not be built")
