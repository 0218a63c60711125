"""Steepest-descent energy minimizer, float64 (oracle).

Test infrastructure only.  Restates MdState::minimize_energy and
step_energy_min (src/minimize_energy.rs:60-260): reciprocal-space forces
off (:96-99), waters and static atoms fixed, each trial moving every atom
by F * step / F_max with step = min(alpha F_max, 0.2 A) (:160-190);
accept when the potential energy does not rise (alpha = min(1.2 alpha,
0.01); converged when the largest force is <= tol, :205-212), else revert
and halve alpha (stop below 1e-8, :214-237).
"""
import numpy as np

from . import method

STEP_MAX = 0.2
GROW = 1.2
SHRINK = 0.5
ALPHA_MIN = 1.0e-8
ALPHA_MAX = 1.0e-2


def minimize_energy(sysd, params, max_iters, tol):
    """Returns (atom positions float64, accepted steps, final energy)."""
    p = dict(params)
    p["recip_disabled"] = True
    x = np.asarray(sysd["atom_pos"], np.float64).copy()
    movable = ~np.asarray(sysd.get("atom_static", np.zeros(len(x), bool)), bool)

    def evaluate(x):
        d = dict(sysd)
        d["atom_pos"] = x
        r = method.all_forces(d, p)
        return r["f_atoms"], r["pe"]

    f, e_prev = evaluate(x)
    alpha = 0.01
    accepted = 0
    for _ in range(max_iters):
        alpha_try = alpha
        while True:
            fm = np.linalg.norm(f, axis=1)
            ok = movable & np.isfinite(fm)
            f_max = float(fm[ok].max()) if ok.any() else 0.0
            if f_max == 0.0:
                return x, accepted, e_prev
            step = min(alpha_try * f_max, STEP_MAX)
            s = np.where((ok & (fm != 0.0))[:, None], f * (step / f_max), 0.0)
            x = x + s
            f_new, e_new = evaluate(x)
            if e_new <= e_prev:
                e_prev = e_new
                alpha = min(alpha_try * GROW, ALPHA_MAX)
                accepted += 1
                f = f_new
                fn = np.linalg.norm(f, axis=1)
                if float(fn[movable & np.isfinite(fn)].max(initial=0.0)) <= tol:
                    return x, accepted, e_prev
                break
            x = x - s
            alpha_try *= SHRINK
            if alpha_try < ALPHA_MIN:
                return x, accepted, e_prev
    return x, accepted, e_prev
