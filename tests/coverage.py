"""Pairs inside the cutoff (periodic k-d trees, float64) and their coverage
by the resident engine's neighbour lists (MdState.list_pairs).

A water pair needs to be evaluated when an interacting site pair lies within
the cutoff: O-O (LJ) or a pair of charged sites (H0, H1, M).  A water-atom
pair needs it when the atom lies within the cutoff of any water site, an
atom pair when it is within the cutoff and is neither an exclusion (1-2,
1-3) nor a 1-4 pair (those are evaluated by their own kernel).
"""
import numpy as np
from scipy.spatial import cKDTree


def _wrap(p, lo, ext):
    x = np.mod(np.asarray(p, np.float64) - lo, ext)
    return np.where(x >= ext, 0.0, x)


def _keys(a, b, n):
    a = np.asarray(a, np.int64)
    b = np.asarray(b, np.int64)
    return np.unique(np.minimum(a, b) * n + np.maximum(a, b))


def needed_pairs(state, sysd, cutoff):
    """(ww, ws, ss) int64 keys of the pairs that must be in the lists."""
    lo = np.asarray(sysd["box_lo"], np.float64)
    ext = (np.asarray(sysd["box_hi"], np.float32) - np.asarray(sysd["box_lo"], np.float32)).astype(np.float64)
    wp = np.asarray(state["water_pos"], np.float64)
    nw = len(wp)
    ap = np.asarray(state["atom_pos"], np.float64).reshape(-1, 3)
    na = len(ap)
    ww = ws = ss = np.zeros(0, np.int64)
    if nw:
        o = _wrap(wp[:, 0], lo, ext)
        ch = _wrap(np.stack([wp[:, 1], wp[:, 2], np.asarray(state["water_m"], np.float64)], axis=1).reshape(-1, 3),
                   lo, ext)
        p_oo = cKDTree(o, boxsize=ext).query_pairs(cutoff, output_type="ndarray")
        p_cc = cKDTree(ch, boxsize=ext).query_pairs(cutoff, output_type="ndarray")
        a, b = p_cc[:, 0] // 3, p_cc[:, 1] // 3
        keep = a != b
        ww = np.unique(np.concatenate([_keys(p_oo[:, 0], p_oo[:, 1], nw), _keys(a[keep], b[keep], nw)]))
    if na:
        at = cKDTree(_wrap(ap, lo, ext), boxsize=ext)
        if nw:
            allw = _wrap(np.concatenate([wp, np.asarray(state["water_m"], np.float64)[:, None]], axis=1)
                         .reshape(-1, 3), lo, ext)
            m = cKDTree(allw, boxsize=ext).sparse_distance_matrix(at, cutoff, output_type="ndarray")
            ws = np.unique(np.asarray(m["i"], np.int64) // 4 * na + np.asarray(m["j"], np.int64))
        p = at.query_pairs(cutoff, output_type="ndarray")
        ss = _keys(p[:, 0], p[:, 1], na)
        skip = [np.asarray(sysd.get(k, np.zeros((0, 2))), np.int64).reshape(-1, 2) for k in ("excl", "pair14")]
        skip = np.concatenate(skip)
        if len(skip):
            ss = np.setdiff1d(ss, _keys(skip[:, 0], skip[:, 1], na))
        st = np.asarray(sysd.get("atom_static", np.zeros(na, bool)), bool)
        if st.any():
            ss = ss[~(st[ss // na] & st[ss % na])]
    return ww, ws, ss


def covered_pairs(st, n_water, n_atoms):
    """(ww, ws, ss) int64 keys of the pairs the engine's lists hold."""
    out = []
    for kind, n, ordered in ((0, n_water, False), (1, n_atoms, True), (2, n_atoms, False)):
        p = st.list_pairs(kind).astype(np.int64)
        if ordered:
            out.append(np.unique(p[:, 0] * n + p[:, 1]))
        else:
            out.append(_keys(p[:, 0], p[:, 1], max(n, 1)))
    return tuple(out)


def missing(needed, covered):
    """Per kind, the needed keys absent from the lists."""
    return [nd[~np.isin(nd, cv)] for nd, cv in zip(needed, covered)]
