"""Neighbour lists, flat pair assembly and short-range pair math (oracle).

Restates, in numpy:

* SimBox::wrap / SimBox::min_image (src/barostat.rs:141-170) in exact float32
  arithmetic (numpy float32 ops are IEEE round-to-nearest with no FMA
  contraction, matching Rust ``f32``);
* build_neighbors / build_all_neighbors (src/neighbors.rs:102-156,180-281):
  brute-force O(N^2) lists with ``|min_image(d)|^2 < (cutoff+skin)^2``;
* setup_pairs (src/non_bonded.rs:541-677) and the per-pair SoA that
  PerNeighborGpu::new uploads (src/gpu_interface.rs:243-410);
* the pair math of f_nonbonded_cpu (src/non_bonded.rs:950-1057) and of the
  GPU twin nonbonded_force_kernel (src/cuda/cuda.cu:185-362), in float64.

The erfc-screened Coulomb form is the one the reference's CUDA kernel states
(src/cuda/cuda.cu:148-180); the CPU path calls the external
``ewald::force_coulomb_short_range`` whose source is absent.
"""
import numpy as np
from scipy.special import erfc

from . import opc

f32 = np.float32

# Water site codes of the reference (src/solvent/mod.rs:256-261).
SITE_O, SITE_M, SITE_H0, SITE_H1 = 1, 2, 3, 4
# Pair-list site iteration order of setup_pairs (src/non_bonded.rs:550).
SITES_ORDER = (SITE_O, SITE_M, SITE_H0, SITE_H1)


# --------------------------------------------------------------------------
# float32-exact SimBox helpers
# --------------------------------------------------------------------------

def round_half_away_f32(q):
    """Rust ``f32::round``: nearest integer, ties away from zero (exact)."""
    q = np.asarray(q, dtype=f32)
    t = np.trunc(q)
    frac = q - t  # exact in float32
    return (t + np.where(np.abs(frac) >= f32(0.5), np.sign(q), f32(0.0))).astype(f32)


def min_image_f32(dv, ext):
    """SimBox::min_image (src/barostat.rs:162-170), float32-exact."""
    dv = np.asarray(dv, dtype=f32)
    ext = np.asarray(ext, dtype=f32)
    q = (dv / ext).astype(f32)
    return (dv - (round_half_away_f32(q) * ext).astype(f32)).astype(f32)


def wrap_f32(p, lo, ext):
    """SimBox::wrap (src/barostat.rs:141-157): rem_euclid, float32-exact."""
    p = np.asarray(p, dtype=f32)
    lo = np.asarray(lo, dtype=f32)
    ext = np.asarray(ext, dtype=f32)
    a = (p - lo).astype(f32)
    r = np.fmod(a, ext).astype(f32)
    r = np.where(r < 0, (r + np.abs(ext)).astype(f32), r).astype(f32)
    return (r + lo).astype(f32)


def mag_sq_f32(d):
    """|d|^2 evaluated left to right in float32: (x*x + y*y) + z*z."""
    d = np.asarray(d, dtype=f32)
    x, y, z = d[..., 0], d[..., 1], d[..., 2]
    return ((x * x + y * y).astype(f32) + z * z).astype(f32)


# --------------------------------------------------------------------------
# neighbour lists
# --------------------------------------------------------------------------

def build_neighbors(posits_outer, posits_inner, is_static, ext, symmetric,
                    skin_sq_w_cutoff, chunk=512):
    """build_neighbors (src/neighbors.rs:180-281).

    Returns a list (one entry per outer index) of ascending int arrays.  For
    ``symmetric`` the half lists (i < j) are computed and mirrored exactly as
    the reference does, which leaves every row sorted ascending.
    """
    po = np.asarray(posits_outer, dtype=f32)
    pi = np.asarray(posits_inner, dtype=f32)
    thr = f32(skin_sq_w_cutoff)
    n_o = po.shape[0]
    n_i = pi.shape[0]
    rows = []
    for s in range(0, n_o, chunk):
        e = min(n_o, s + chunk)
        d = min_image_f32(po[s:e, None, :] - pi[None, :, :], ext)
        hit = mag_sq_f32(d) < thr
        if symmetric:
            idx = np.arange(n_i)[None, :]
            hit &= idx > np.arange(s, e)[:, None]
            if is_static is not None:
                st = np.asarray(is_static, dtype=bool)
                hit &= ~(st[s:e, None] & st[None, :])
        for r in range(e - s):
            rows.append(np.nonzero(hit[r])[0])
    if not symmetric:
        return rows
    full = [[] for _ in range(n_o)]
    for i in range(n_o):
        for j in rows[i]:
            full[i].append(j)
            full[int(j)].append(i)
    return [np.array(sorted(r), dtype=np.int64) for r in full]


def build_all_neighbors(sysd, skin, cutoff):
    """build_all_neighbors (src/neighbors.rs:102-156): three lists."""
    lo = np.asarray(sysd["box_lo"], dtype=f32)
    hi = np.asarray(sysd["box_hi"], dtype=f32)
    ext = (hi - lo).astype(f32)
    thr = f32((f32(cutoff) + f32(skin)) * (f32(cutoff) + f32(skin)))
    atom_pos = np.asarray(sysd["atom_pos"], dtype=f32).reshape(-1, 3)
    water_o = np.asarray(sysd["water_pos"], dtype=f32).reshape(-1, 3, 3)[:, 0, :]
    water_o_wrapped = wrap_f32(water_o, lo, ext)
    is_static = np.asarray(sysd.get("atom_static", np.zeros(len(atom_pos), bool)), dtype=bool)
    std_std = build_neighbors(atom_pos, atom_pos, is_static, ext, True, thr)
    std_water = build_neighbors(atom_pos, water_o_wrapped, None, ext, False, thr)
    water_water = build_neighbors(water_o_wrapped, water_o_wrapped, None, ext, True, thr)
    return std_std, std_water, water_water


# --------------------------------------------------------------------------
# flat pair list (setup_pairs + PerNeighborGpu layout)
# --------------------------------------------------------------------------

def setup_pairs(sysd, lists, alch_range=None):
    """setup_pairs (src/non_bonded.rs:541-677) flattened to the SoA that
    PerNeighborGpu::new builds (src/gpu_interface.rs:243-340).

    ``alch_range`` = (begin, end): the alchemical molecule's atoms; the
    ``alch`` column flags atom-atom pairs with exactly one end inside and
    atom-water pairs whose atom is inside (src/non_bonded.rs:581-612).

    Returns a dict of numpy arrays, one entry per pair, in the reference's
    canonical order: std-std (i<j), std-water (sites O,M,H0,H1), water-water
    (i0<i1, the 10 (site0, site1) combinations with LJ or Coulomb).
    """
    std_std, std_water, water_water = lists
    n_std = len(std_std)
    excl = set(map(tuple, np.asarray(sysd.get("excl", np.zeros((0, 2))), dtype=np.int64).tolist()))
    s14 = set(map(tuple, np.asarray(sysd.get("pair14", np.zeros((0, 2))), dtype=np.int64).tolist()))
    bonded_only = np.asarray(sysd.get("atom_bonded_only", np.zeros(n_std, bool)), dtype=bool)
    sig = np.asarray(sysd.get("atom_sigma", np.zeros(n_std)), dtype=f32)
    eps = np.asarray(sysd.get("atom_eps", np.zeros(n_std)), dtype=f32)
    q_atom = np.asarray(sysd.get("atom_q", np.zeros(n_std)), dtype=f32)
    site_q = {SITE_O: f32(0.0), SITE_M: opc.Q_EP, SITE_H0: opc.Q_H, SITE_H1: opc.Q_H}

    cols = {k: [] for k in ("tgt", "src", "sigma", "eps", "q_tgt", "q_src", "atype_tgt",
                            "wtype_tgt", "atype_src", "wtype_src", "scale_14", "calc_lj",
                            "calc_coulomb", "symmetric", "alch")}
    ab, ae = alch_range if alch_range is not None else (0, 0)

    def in_alch(i):
        return ab <= i < ae

    def push(t, s, sg, ep, qt, qs, at, wt, as_, ws, sc, lj, co, al=0):
        cols["alch"].append(al)
        cols["tgt"].append(t); cols["src"].append(s)
        cols["sigma"].append(sg); cols["eps"].append(ep)
        cols["q_tgt"].append(qt); cols["q_src"].append(qs)
        cols["atype_tgt"].append(at); cols["wtype_tgt"].append(wt)
        cols["atype_src"].append(as_); cols["wtype_src"].append(ws)
        cols["scale_14"].append(sc); cols["calc_lj"].append(lj)
        cols["calc_coulomb"].append(co); cols["symmetric"].append(1)

    # std-std (src/non_bonded.rs:565-599); LJ mixing src/non_bonded.rs:1081-1086
    for i in range(n_std):
        for j in std_std[i]:
            j = int(j)
            if j <= i:
                continue
            if bonded_only[i] or bonded_only[j]:
                continue
            if (i, j) in excl:
                continue
            sg = f32(f32(0.5) * (sig[i] + sig[j]))
            ep = f32(np.sqrt(f32(eps[i] * eps[j]), dtype=f32))
            push(i, j, sg, ep, q_atom[i], q_atom[j], 0, 0, 0, 0, int((i, j) in s14), 1, 1,
                 int(in_alch(i) != in_alch(j)))
    # std-water (src/non_bonded.rs:605-625); LJ row src/non_bonded.rs:139-145
    for i in range(n_std):
        sg = f32(f32(0.5) * (sig[i] + opc.O_SIGMA))
        ep = f32(np.sqrt(f32(eps[i] * opc.O_EPS), dtype=f32))
        for w in std_water[i]:
            for site in SITES_ORDER:
                push(i, int(w), sg, ep, q_atom[i], site_q[site], 0, 0, 1, site, 0,
                     int(site == SITE_O), int(site != SITE_O), int(in_alch(i)))
    # water-water (src/non_bonded.rs:628-664)
    for i0 in range(len(water_water)):
        for i1 in water_water[i0]:
            i1 = int(i1)
            if i1 <= i0:
                continue
            for s0 in SITES_ORDER:
                for s1 in SITES_ORDER:
                    lj = s0 == SITE_O and s1 == SITE_O
                    co = s0 != SITE_O and s1 != SITE_O
                    if not (lj or co):
                        continue
                    push(i0, i1, opc.O_SIGMA, opc.O_EPS, site_q[s0], site_q[s1], 1, s0, 1, s1,
                         0, int(lj), int(co))
    out = {}
    for k, v in cols.items():
        if k in ("tgt", "src"):
            out[k] = np.asarray(v, dtype=np.uint32)
        elif k in ("sigma", "eps", "q_tgt", "q_src"):
            out[k] = np.asarray(v, dtype=f32)
        else:
            out[k] = np.asarray(v, dtype=np.uint8)
    return out


# --------------------------------------------------------------------------
# pair math
# --------------------------------------------------------------------------

def site_positions(sysd):
    """(pos_dyn, {site: pos}) as float32, with M from the virtual-site rule."""
    wp = np.asarray(sysd["water_pos"], dtype=f32).reshape(-1, 3, 3)
    if "water_m" in sysd:
        m = np.asarray(sysd["water_m"], dtype=f32).reshape(-1, 3)
    else:
        m = opc.virtual_site(wp[:, 0].astype(np.float64), wp[:, 1].astype(np.float64),
                             wp[:, 2].astype(np.float64)).astype(f32)
    return (np.asarray(sysd["atom_pos"], dtype=f32).reshape(-1, 3),
            {SITE_O: wp[:, 0], SITE_M: m, SITE_H0: wp[:, 1], SITE_H1: wp[:, 2]})


def _gather(pos_dyn, pos_w, atype, wtype, idx):
    out = np.zeros((len(idx), 3), dtype=np.float64)
    dyn = atype == 0
    out[dyn] = pos_dyn[idx[dyn]]
    for s in SITES_ORDER:
        sel = (atype == 1) & (wtype == s)
        out[sel] = pos_w[s][idx[sel]]
    return out


def pair_forces(pairs, pos_dyn, pos_w, ext, cutoff, alpha, lj_cutoff=None,
                lj_disabled=False, coulomb_disabled=False, gpu_semantics=False,
                lambda_alch=None):
    """Per-pair force on the target, energy and virial in float64.

    With ``lambda_alch`` given, pairs whose ``alch`` column is set take
    soft-core LJ and scaled Coulomb on the staged decoupling schedule
    (nonbonded_force_alchemical_kernel, src/cuda/cuda.cu:367-566;
    f_nonbonded_cpu, src/non_bonded.rs:950-1057) and the function returns
    a fifth value, their summed dH/dlambda.

    ``gpu_semantics`` selects the reference CUDA kernel's conventions
    (src/cuda/cuda.cu:239-316): no LJ cutoff, r^2 < 1e-16 skip, energy only
    for non-water targets.  Otherwise the CPU conventions of f_nonbonded_cpu
    (src/non_bonded.rs:967-1054, src/non_bonded.rs:335-342): LJ only for
    r <= lj_cutoff, r^2 < 1e-12 skip, energy when either body is non-water.
    Coulomb is zero for r >= cutoff in both.
    """
    pt = _gather(pos_dyn, pos_w, pairs["atype_tgt"], pairs["wtype_tgt"], pairs["tgt"].astype(np.int64))
    ps = _gather(pos_dyn, pos_w, pairs["atype_src"], pairs["wtype_src"], pairs["src"].astype(np.int64))
    ext = np.asarray(ext, dtype=np.float64)
    d = pt - ps
    d = d - np.round(d / ext) * ext
    r2 = np.einsum("ij,ij->i", d, d)
    skip = r2 < (1e-16 if gpu_semantics else 1e-12)
    r2s = np.where(skip, 1.0, r2)
    r = np.sqrt(r2s)
    inv_r = 1.0 / r
    sig = pairs["sigma"].astype(np.float64)
    eps = pairs["eps"].astype(np.float64)
    sr6 = (sig * inv_r) ** 6
    f_lj = 24.0 * eps * (2.0 * sr6 * sr6 - sr6) * inv_r
    e_lj = 4.0 * eps * (sr6 * sr6 - sr6)
    lj_on = pairs["calc_lj"].astype(bool) & (not lj_disabled)
    if not gpu_semantics:
        lj_c = cutoff if lj_cutoff is None else lj_cutoff
        lj_on &= r <= lj_c
    qq = pairs["q_tgt"].astype(np.float64) * pairs["q_src"].astype(np.float64)
    ar = alpha * r
    f_c = qq * (erfc(ar) * inv_r * inv_r + 2.0 * alpha / np.sqrt(np.pi) * np.exp(-ar * ar) * inv_r)
    e_c = qq * erfc(ar) * inv_r
    co_on = pairs["calc_coulomb"].astype(bool) & (not coulomb_disabled) & (r < cutoff)
    f_lj = np.where(lj_on, f_lj, 0.0)
    e_lj = np.where(lj_on, e_lj, 0.0)
    f_c = np.where(co_on, f_c, 0.0)
    e_c = np.where(co_on, e_c, 0.0)
    sc = pairs["scale_14"].astype(bool)
    f_lj = np.where(sc, f_lj * 0.5, f_lj)
    e_lj = np.where(sc, e_lj * 0.5, e_lj)
    f_c = np.where(sc, f_c / 1.2, f_c)
    e_c = np.where(sc, e_c / 1.2, e_c)
    dh = np.zeros(len(r))
    alch = None
    if lambda_alch is not None and "alch" in pairs:
        from .method import decoupling_schedule, soft_core_lj
        cs, dcs, ll, dll = decoupling_schedule(np.float32(lambda_alch))
        alch = pairs["alch"].astype(bool)
        # the CPU path evaluates a coincident alchemical pair at r = 0
        r_sc = np.where(skip, 0.0, r)
        fs, es, dv = _soft_core_at(r_sc, sig, eps, ll, soft_core_lj)
        # pairs with LJ soft-core terms: the evaluated ones, plus (CPU path
        # only) coincident pairs, which keep their contact energy
        lj_sc = (lj_on & ~skip) | (skip & ~np.bool_(gpu_semantics) & pairs["calc_lj"].astype(bool)
                                   & (not lj_disabled))
        w14 = np.where(sc, 0.5, 1.0)
        f_lj = np.where(alch, np.where(lj_on, fs * w14, 0.0), f_lj)
        e_lj = np.where(alch, np.where(lj_sc, es * w14, 0.0), e_lj)
        dh = np.where(alch & lj_sc, dv * dll * w14, 0.0)
        dh = dh + np.where(alch & ~skip, e_c * dcs, 0.0)
        f_c = np.where(alch, f_c * cs, f_c)
        e_c = np.where(alch, e_c * cs, e_c)
    fmag = np.where(skip, 0.0, f_lj + f_c)
    e = np.where(skip, 0.0, e_lj + e_c)
    if alch is not None and not gpu_semantics:
        e = np.where(skip & alch, e_lj, e)
    f = d * (fmag * inv_r)[:, None]
    virial = float(np.sum(fmag * r))
    if gpu_semantics:
        e_mask = pairs["atype_tgt"] == 0
    else:
        e_mask = (pairs["atype_tgt"] == 0) | (pairs["atype_src"] == 0)
    energy = float(np.sum(e[e_mask]))
    if lambda_alch is not None:
        return f, energy, virial, e, float(np.sum(dh))
    return f, energy, virial, e


def _soft_core_at(r, sig, eps, lam, soft_core_lj):
    """soft_core_lj with the reference's guards: zero where eps is 0 or the
    soft-core radius is 0 (r = 0 at lambda 0)."""
    ss6 = np.maximum(sig, 3.0) ** 6
    ok = (eps != 0.0) & (r ** 6 + 0.5 * ss6 * lam > 0.0)
    fs, es, dv = soft_core_lj(np.where(ok, r, 1.0), sig, np.where(ok, eps, 0.0), lam)
    return np.where(ok, fs, 0.0), np.where(ok, es, 0.0), np.where(ok, dv, 0.0)


def accumulate_pair_forces(pairs, f, n_dyn, n_water):
    """Scatter per-pair target forces (and the mirrored source forces of
    symmetric pairs) into dyn and per-site water arrays, as
    calc_force_cpu's add_to_sink does (src/non_bonded.rs:235-251,330-333)."""
    f_dyn = np.zeros((n_dyn, 3))
    f_w = {s: np.zeros((n_water, 3)) for s in SITES_ORDER}
    for side, sign in (("tgt", 1.0), ("src", -1.0)):
        at = pairs["atype_" + side]
        wt = pairs["wtype_" + side]
        idx = pairs[side].astype(np.int64)
        sel_sym = np.ones(len(idx), bool) if side == "tgt" else pairs["symmetric"].astype(bool)
        dyn = (at == 0) & sel_sym
        np.add.at(f_dyn, idx[dyn], sign * f[dyn])
        for s in SITES_ORDER:
            sel = (at == 1) & (wt == s) & sel_sym
            np.add.at(f_w[s], idx[sel], sign * f[sel])
    return f_dyn, f_w


def lj_force_energy(inv_dist, sigma, eps):
    """force_e_lj (src/forces.rs:10-21): magnitude along dir and energy."""
    sr = sigma * inv_dist
    sr6 = sr ** 6
    sr12 = sr6 * sr6
    return 24.0 * eps * (2.0 * sr12 - sr6) * inv_dist, 4.0 * eps * (sr12 - sr6)


def coulomb_short_range(dist, q0, q1, cutoff, alpha):
    """Magnitude along dir and energy of the erfc-screened Coulomb term
    (src/cuda/cuda.cu:148-180); zero for dist >= cutoff."""
    dist = np.asarray(dist, dtype=np.float64)
    inv = 1.0 / dist
    ar = alpha * dist
    f = q0 * q1 * (erfc(ar) * inv * inv + 2.0 * alpha / np.sqrt(np.pi) * np.exp(-ar * ar) * inv)
    e = q0 * q1 * erfc(ar) * inv
    inside = dist < cutoff
    return np.where(inside, f, 0.0), np.where(inside, e, 0.0)
