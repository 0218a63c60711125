"""Full FP64 force evaluation of the engine's method (oracle).

One call restates MdState::reset_f_acc_pe_virial + apply_all_forces
(src/lib.rs:1220-1348) for a system dict, independently of any neighbour
list: every site pair within the cutoff is found with a periodic k-d tree,
so the result is the method's answer, not the answer of a particular list.

Semantics (shared with the CUDA engine):

* short range -- LJ between sites that carry LJ (solute atoms, water O) for
  r <= lj_cutoff; erfc-screened Coulomb between charged sites (solute atoms,
  water M/H0/H1) for r < coulomb_cutoff (f_nonbonded_cpu,
  src/non_bonded.rs:950-1057).  Intra-water pairs and 1-2/1-3 exclusions are
  skipped; 1-4 pairs are scaled LJ x0.5, Coulomb x1/1.2
  (src/non_bonded.rs:55-56,565-599).
* reciprocal -- SPME over all charged sites, wrapped into the box
  (src/non_bonded.rs:681-846), energy including the self term.
* ``reference`` mode reproduces the reference's bookkeeping: no exclusion
  correction in k-space, the 1-4 vacuum force correction
  (src/non_bonded.rs:763-790), and a potential energy that omits
  water-water real-space energy (src/non_bonded.rs:335-342).
* ``corrected`` mode adds the Ewald exclusion correction (-q q erf(ar)/r for
  intra-water and 1-2/1-3 pairs, -(1/6) q q erf(ar)/r for 1-4 pairs) and
  counts every energy term.
* bonded terms follow src/bonded.rs:23-135 and src/bonded_forces.rs.
"""
import numpy as np
from scipy.spatial import cKDTree
from scipy.special import erfc, erf

from . import opc, spme
from . import bonded as bonded_mod

W_O, W_H0, W_H1, W_M = 0, 1, 2, 3


def water_sites(sysd):
    """(nw, 4, 3) float64 site positions in engine order O, H0, H1, M."""
    wp = np.asarray(sysd["water_pos"], dtype=np.float32).reshape(-1, 3, 3).astype(np.float64)
    if "water_m" in sysd:
        m = np.asarray(sysd["water_m"], dtype=np.float32).reshape(-1, 3).astype(np.float64)
    else:
        m = opc.virtual_site(wp[:, 0], wp[:, 1], wp[:, 2])
        m = m.astype(np.float32).astype(np.float64)
    return np.concatenate([wp, m[:, None, :]], axis=1)


def _site_tables(sysd):
    na = len(np.asarray(sysd["atom_pos"]).reshape(-1, 3))
    ws = water_sites(sysd)
    nw = ws.shape[0]
    pos = np.concatenate([np.asarray(sysd["atom_pos"], dtype=np.float32).reshape(-1, 3).astype(np.float64),
                          ws.reshape(-1, 3)], axis=0)
    q = np.concatenate([np.asarray(sysd.get("atom_q", np.zeros(na)), dtype=np.float32).astype(np.float64),
                        np.tile(np.array([0.0, float(opc.Q_H), float(opc.Q_H), float(opc.Q_EP)]), nw)])
    sig = np.concatenate([np.asarray(sysd.get("atom_sigma", np.zeros(na)), dtype=np.float32).astype(np.float64),
                          np.tile(np.array([float(opc.O_SIGMA), 0, 0, 0]), nw)])
    eps = np.concatenate([np.asarray(sysd.get("atom_eps", np.zeros(na)), dtype=np.float32).astype(np.float64),
                          np.tile(np.array([float(opc.O_EPS), 0, 0, 0]), nw)])
    has_lj = np.concatenate([np.ones(na, bool), np.tile(np.array([True, False, False, False]), nw)])
    mol = np.concatenate([-1 - np.arange(na), np.repeat(np.arange(nw), 4)])
    return pos, q, sig, eps, has_lj, mol, na, nw


def decoupling_schedule(lam):
    """staged_decoupling_schedule (src/alchemical.rs:77-96): (Coulomb scale,
    its lambda derivative, LJ soft-core lambda, its lambda derivative)."""
    lam = min(max(float(lam), 0.0), 1.0)
    if lam < 0.5:
        return 1.0 - 2.0 * lam, -2.0, 0.0, 0.0
    return 0.0, 0.0, 2.0 * lam - 1.0, 2.0


SC_ALPHA, SC_SIGMA_MIN = 0.5, 3.0  # src/alchemical.rs:55-65 (power 1)


def soft_core_lj(r, sig, eps, lam):
    """alchemical_lj_soft_core_decouple (src/non_bonded.rs:883-941) per
    pair: (force magnitude along r, energy, dV/dl)."""
    ss6 = np.maximum(sig, SC_SIGMA_MIN) ** 6
    rsc6 = r ** 6 + SC_ALPHA * ss6 * lam
    rsc = rsc6 ** (1.0 / 6.0)
    sr6 = (sig / rsc) ** 6
    hf = 24.0 * eps * (2.0 * sr6 * sr6 - sr6) / rsc
    he = 4.0 * eps * (sr6 * sr6 - sr6)
    scale = 1.0 - lam
    fmag = hf * scale * (r / rsc) ** 5
    dvdl = -he - scale * hf * SC_ALPHA * ss6 / (6.0 * rsc ** 5)
    return np.where(eps != 0.0, fmag, 0.0), np.where(eps != 0.0, scale * he, 0.0), np.where(eps != 0.0, dvdl, 0.0)


def short_range(sysd, cutoff, alpha, lj_cutoff=None, lj_disabled=False, coulomb_disabled=False, alch=None):
    """Short-range forces over all site pairs within the cutoff (FP64).

    Returns dict with per-site forces (n_sites, 3), energy split into
    water-water and solute-involving parts, virial and the pair count.
    Sites are ordered atoms first, then water O, H0, H1, M per molecule.
    ``alch`` = (begin, end, lambda): pairs with exactly one atom in
    [begin, end) take soft-core LJ and scaled Coulomb on the staged schedule
    (f_nonbonded_cpu, src/non_bonded.rs:950-1057); their dH/dlambda is
    returned as ``dh_dl``.
    """
    pos, q, sig, eps, has_lj, mol, na, nw = _site_tables(sysd)
    lo = np.asarray(sysd["box_lo"], dtype=np.float32).astype(np.float64)
    ext = (np.asarray(sysd["box_hi"], dtype=np.float32) - np.asarray(sysd["box_lo"], dtype=np.float32)).astype(np.float64)
    lj_c = cutoff if lj_cutoff is None else lj_cutoff
    rmax = max(cutoff, lj_c)
    assert rmax < 0.5 * ext.min(), "cutoff must be below half the box"
    wrapped = np.mod(pos - lo, ext)
    wrapped = np.where(wrapped >= ext, 0.0, wrapped)
    tree = cKDTree(wrapped, boxsize=ext)
    pairs = tree.query_pairs(rmax * (1 + 1e-9) + 1e-9, output_type="ndarray")
    i, j = pairs[:, 0], pairs[:, 1]
    keep = ~((mol[i] == mol[j]) & (mol[i] >= 0))  # no intra-water pairs
    i, j = i[keep], j[keep]
    excl = np.asarray(sysd.get("excl", np.zeros((0, 2))), dtype=np.int64).reshape(-1, 2)
    p14 = np.asarray(sysd.get("pair14", np.zeros((0, 2))), dtype=np.int64).reshape(-1, 2)
    scale = np.ones(len(i))
    lj_scale = np.ones(len(i))
    if len(excl) or len(p14):
        key = np.minimum(i, j) * (na + 1) + np.maximum(i, j)
        both_atoms = (i < na) & (j < na)
        if len(excl):
            ek = np.minimum(excl[:, 0], excl[:, 1]) * (na + 1) + np.maximum(excl[:, 0], excl[:, 1])
            drop = both_atoms & np.isin(key, ek)
            i, j, key, both_atoms = i[~drop], j[~drop], key[~drop], both_atoms[~drop]
            scale, lj_scale = scale[~drop], lj_scale[~drop]
        if len(p14):
            pk = np.minimum(p14[:, 0], p14[:, 1]) * (na + 1) + np.maximum(p14[:, 0], p14[:, 1])
            is14 = both_atoms & np.isin(key, pk)
            scale = np.where(is14, 1.0 / 1.2, scale)
            lj_scale = np.where(is14, 0.5, lj_scale)
    d = pos[i] - pos[j]
    d = d - np.round(d / ext) * ext
    r2 = np.sum(d * d, axis=1)
    r = np.sqrt(r2)
    inv_r = 1.0 / r
    sg = 0.5 * (sig[i] + sig[j])
    ep = np.sqrt(eps[i] * eps[j])
    sr6 = (sg * inv_r) ** 6
    lj_on = has_lj[i] & has_lj[j] & (r <= lj_c) & (not lj_disabled)
    f_lj = np.where(lj_on, 24.0 * ep * (2.0 * sr6 * sr6 - sr6) * inv_r, 0.0) * lj_scale
    e_lj = np.where(lj_on, 4.0 * ep * (sr6 * sr6 - sr6), 0.0) * lj_scale
    qq = q[i] * q[j]
    co_on = (qq != 0.0) & (r < cutoff) & (not coulomb_disabled)
    ar = alpha * r
    f_c = np.where(co_on, qq * (erfc(ar) * inv_r * inv_r
                                + 2.0 * alpha / np.sqrt(np.pi) * np.exp(-ar * ar) * inv_r), 0.0) * scale
    e_c = np.where(co_on, qq * erfc(ar) * inv_r, 0.0) * scale
    dh_dl = 0.0
    if alch is not None:
        a0, a1, lam = alch
        cs, dcs, ll, dll = decoupling_schedule(lam)
        in_i = (i < na) & (i >= a0) & (i < a1)
        in_j = (j < na) & (j >= a0) & (j < a1)
        cross = in_i != in_j
        fs, es, dv = soft_core_lj(r, sg, ep, ll)
        f_lj = np.where(cross, np.where(lj_on, fs, 0.0), f_lj)
        e_lj = np.where(cross, np.where(lj_on, es, 0.0), e_lj)
        dh_dl = float(np.sum(np.where(cross & lj_on, dv, 0.0))) * dll
        dh_dl += float(np.sum(np.where(cross, e_c, 0.0))) * dcs
        f_c = np.where(cross, f_c * cs, f_c)
        e_c = np.where(cross, e_c * cs, e_c)
    fmag = f_lj + f_c
    f = d * (fmag * inv_r)[:, None]
    n = len(pos)
    forces = np.zeros((n, 3))
    np.add.at(forces, i, f)
    np.add.at(forces, j, -f)
    ww = (i >= na) & (j >= na)
    e = e_lj + e_c
    return {
        "forces": forces,
        "e_lj": float(np.sum(e_lj)),
        "e_coul": float(np.sum(e_c)),
        "e_water_water": float(np.sum(e[ww])),
        "e_solute": float(np.sum(e[~ww])),
        "virial": float(np.sum(fmag * r)),
        "n_lj_pairs": int(np.count_nonzero(lj_on)),
        "n_coul_pairs": int(np.count_nonzero(co_on)),
        "n_pairs_within": int(np.count_nonzero(lj_on | co_on)),
        "na": na, "nw": nw, "dh_dl": dh_dl,
    }


def charged_sites(sysd):
    """Charged site positions, wrapped into the box, and charges, in
    pack_pme_pos_q order (src/non_bonded.rs:800-826): atoms, then M, H0, H1
    per water."""
    pos, q, sig, eps, has_lj, mol, na, nw = _site_tables(sysd)
    lo = np.asarray(sysd["box_lo"], dtype=np.float32).astype(np.float64)
    ext = (np.asarray(sysd["box_hi"], dtype=np.float32) - np.asarray(sysd["box_lo"], dtype=np.float32)).astype(np.float64)
    atoms = pos[:na]
    ws = pos[na:].reshape(nw, 4, 3)
    wq = np.stack([ws[:, W_M], ws[:, W_H0], ws[:, W_H1]], axis=1).reshape(-1, 3)
    p = np.concatenate([atoms, wq], axis=0)
    qq = np.concatenate([q[:na], np.tile(np.array([float(opc.Q_EP), float(opc.Q_H), float(opc.Q_H)]), nw)])
    p = lo + np.mod(p - lo, ext)
    return p, qq, na, nw


def all_forces(sysd, cfg):
    """FP64 forces and energies for one evaluation.

    ``cfg`` keys: cutoff, alpha, grid, lj_cutoff (optional), mode
    ('reference' or 'corrected'), lj_disabled, coulomb_disabled,
    recip_disabled, bonded_disabled.
    Returns dict with 'f_atoms' (na,3), 'f_water' (nw,4,3) [O,H0,H1,M] and
    energy/virial components.
    """
    cutoff = float(cfg["cutoff"])
    alpha = float(cfg["alpha"])
    mode = cfg.get("mode", "reference")
    alch = None
    if cfg.get("alch_range") is not None:
        alch = (int(cfg["alch_range"][0]), int(cfg["alch_range"][1]), float(cfg.get("alch_lambda", 0.0)))
    sr = short_range(sysd, cutoff, alpha, cfg.get("lj_cutoff"), cfg.get("lj_disabled", False),
                     cfg.get("coulomb_disabled", False), alch)
    dh_dl = sr["dh_dl"]
    na, nw = sr["na"], sr["nw"]
    forces = sr["forces"].copy()
    out = {"e_lj": sr["e_lj"], "e_coul_short": sr["e_coul"], "e_water_water_short": sr["e_water_water"],
           "e_solute_short": sr["e_solute"], "virial_short": sr["virial"],
           "n_pairs_within": sr["n_pairs_within"]}
    lo = np.asarray(sysd["box_lo"], dtype=np.float32).astype(np.float64)
    ext = (np.asarray(sysd["box_hi"], dtype=np.float32) - np.asarray(sysd["box_lo"], dtype=np.float32)).astype(np.float64)
    e_recip = 0.0
    w_recip = 0.0
    e_corr = 0.0
    w_corr = 0.0
    if not cfg.get("recip_disabled", False) and not cfg.get("coulomb_disabled", False):
        p, qq, _, _ = charged_sites(sysd)
        if alch is None:
            e_recip, f_rec, w_recip = spme.recip(p, qq, lo, ext, cfg["grid"], alpha, include_self=True)
        else:
            # full, environment-only and molecule-only charges; the cross
            # term scaled (src/non_bonded.rs:709-743)
            a0, a1, lam = alch
            cs, dcs, _, _ = decoupling_schedule(lam)
            mol = np.zeros(len(qq), bool)
            mol[a0:a1] = True
            ef, ff, wf = spme.recip(p, qq, lo, ext, cfg["grid"], alpha, include_self=True)
            ee, fe, we = spme.recip(p, np.where(mol, 0.0, qq), lo, ext, cfg["grid"], alpha, include_self=True)
            em, fm_, wm = spme.recip(p, np.where(mol, qq, 0.0), lo, ext, cfg["grid"], alpha, include_self=True)
            e_recip = ee + em + cs * (ef - ee - em)
            f_rec = fe + fm_ + cs * (ff - fe - fm_)
            w_recip = we + wm + cs * (wf - we - wm)
            dh_dl += dcs * (ef - ee - em)
        forces[:na] += f_rec[:na]
        fw = f_rec[na:].reshape(nw, 3, 3)  # M, H0, H1
        fsite = forces[na:].reshape(nw, 4, 3)
        fsite[:, W_M] += fw[:, 0]
        fsite[:, W_H0] += fw[:, 1]
        fsite[:, W_H1] += fw[:, 2]
        pos_all = np.concatenate([np.asarray(sysd["atom_pos"], dtype=np.float32).reshape(-1, 3).astype(np.float64),
                                  water_sites(sysd).reshape(-1, 3)], axis=0)
        q_atom = np.asarray(sysd.get("atom_q", np.zeros(na)), dtype=np.float32).astype(np.float64)
        p14 = np.asarray(sysd.get("pair14", np.zeros((0, 2))), dtype=np.int64).reshape(-1, 2)
        if mode == "reference":
            # 1-4 vacuum correction (src/non_bonded.rs:763-790)
            if len(p14):
                d = pos_all[p14[:, 0]] - pos_all[p14[:, 1]]
                d = d - np.round(d / ext) * ext
                r = np.sqrt(np.sum(d * d, axis=1))
                dirv = d / r[:, None]
                fv = dirv * (q_atom[p14[:, 0]] * q_atom[p14[:, 1]] / (r * r))[:, None]
                df = fv * (float(opc.SCALE_COUL_14) - 1.0)
                np.add.at(forces, p14[:, 0], df)
                np.add.at(forces, p14[:, 1], -df)
                w_corr += float(np.sum(np.sum(d * df, axis=1)))
        else:
            # Ewald exclusion corrections: intra-water pairs and 1-2/1-3, 1-4.
            ws = water_sites(sysd)
            wq = np.array([0.0, float(opc.Q_H), float(opc.Q_H), float(opc.Q_EP)])
            for a, b in ((W_H0, W_H1), (W_H0, W_M), (W_H1, W_M)):
                e, f, w = spme.exclusion_correction(ws[:, a], ws[:, b], np.full(nw, wq[a]),
                                                    np.full(nw, wq[b]), ext, alpha)
                fsite = forces[na:].reshape(nw, 4, 3)
                fsite[:, a] += f
                fsite[:, b] -= f
                e_corr += e
                w_corr += w
            excl = np.asarray(sysd.get("excl", np.zeros((0, 2))), dtype=np.int64).reshape(-1, 2)
            for lst, sc in ((excl, 1.0), (p14, 1.0 - float(opc.SCALE_COUL_14))):
                if len(lst) == 0:
                    continue
                e, f, w = spme.exclusion_correction(pos_all[lst[:, 0]], pos_all[lst[:, 1]],
                                                    q_atom[lst[:, 0]], q_atom[lst[:, 1]], ext, alpha, sc)
                np.add.at(forces, lst[:, 0], f)
                np.add.at(forces, lst[:, 1], -f)
                e_corr += e
                w_corr += w
    out["e_recip"] = e_recip
    out["virial_recip"] = w_recip
    out["e_excl_corr"] = e_corr
    out["virial_corr"] = w_corr
    e_b = 0.0
    w_b = 0.0
    if not cfg.get("bonded_disabled", False) and na > 0:
        fb, e_b, w_b = bonded_mod.bonded_forces(sysd, ext)
        forces[:na] += fb
    out["e_bonded"] = e_b
    out["virial_bonded"] = w_b
    if mode == "reference":
        out["pe"] = sr["e_solute"] + e_recip + e_b
    else:
        out["pe"] = sr["e_lj"] + sr["e_coul"] + e_recip + e_corr + e_b
    out["virial"] = sr["virial"] + w_recip + w_corr + w_b
    out["f_atoms"] = forces[:na]
    out["f_water"] = forces[na:].reshape(nw, 4, 3)
    out["dh_dl"] = dh_dl
    return out
