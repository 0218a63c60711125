"""Thermodynamic integration over alchemical lambda windows, from the
dH/dlambda the engine records in its snapshot frames (the host-side helpers
of src/alchemical.rs: LambdaWindow, collect_window, free_energy_ti,
free_energy_ti_with_sem, mean_coupled_interaction_kcal).

A window is one run at a fixed lambda: MdConfig(alch_range=..., alch_lambda=l)
or MdState.set_lambda(l), snapshots on, and collect_window(l, frames) on the
frames read back."""
from dataclasses import dataclass

import numpy as np


class AlchemicalError(ValueError):
    pass


@dataclass
class LambdaWindow:
    lam: float
    mean_dh_dl: float   # kcal/mol
    sem_dh_dl: float    # standard error of the mean


@dataclass
class TiEstimate:
    free_energy: float      # kcal/mol
    standard_error: float


def collect_window(lam, frames):
    """Mean and standard error of dH/dlambda over the frames of one window
    (src/alchemical.rs collect_window); frames without a dh_dl are skipped."""
    x = np.array([f["dh_dl"] for f in frames if f.get("dh_dl") is not None], np.float64)
    if len(x) == 0:
        raise AlchemicalError("no dH/dlambda samples")
    if not np.all(np.isfinite(x)):
        raise AlchemicalError(f"non-finite dH/dlambda at lambda {lam}")
    mean = float(x.mean())
    sem = float(np.sqrt(x.var(ddof=1) / len(x))) if len(x) > 1 else float("nan")
    return LambdaWindow(float(lam), mean, sem)


def _check(windows):
    if len(windows) < 2:
        raise AlchemicalError(f"need at least 2 lambda windows, got {len(windows)}")
    for w in windows:
        if not np.isfinite(w.mean_dh_dl):
            raise AlchemicalError(f"non-finite mean dH/dlambda at lambda {w.lam}")
    for a, b in zip(windows, windows[1:]):
        if b.lam <= a.lam:
            raise AlchemicalError(f"lambda windows must be strictly increasing, got {a.lam} followed by {b.lam}")


def free_energy_ti(windows):
    """Trapezoidal integral of the mean dH/dlambda over the (ascending)
    windows, kcal/mol (src/alchemical.rs free_energy_ti)."""
    _check(windows)
    return float(sum(0.5 * (a.mean_dh_dl + b.mean_dh_dl) * (b.lam - a.lam) for a, b in zip(windows, windows[1:])))


def free_energy_ti_with_sem(windows):
    """The integral with its standard error, each interval contributing
    (dlambda / 2)^2 (sem_a^2 + sem_b^2) to the variance, as the reference
    propagates it."""
    g = free_energy_ti(windows)
    var = sum((0.5 * (b.lam - a.lam)) ** 2 * (a.sem_dh_dl ** 2 + b.sem_dh_dl ** 2)
              for a, b in zip(windows, windows[1:]))
    return TiEstimate(g, float(np.sqrt(var)))


def mean_coupled_interaction_kcal(frames):
    """Mean of -dH/dlambda over frames with a finite, non-zero value (a
    lambda = 0 run: the molecule's interaction with its environment, more
    negative = stronger attraction); None without samples."""
    x = [-f["dh_dl"] for f in frames if f.get("dh_dl") is not None and np.isfinite(f["dh_dl"]) and f["dh_dl"] != 0.0]
    return float(np.mean(x)) if x else None
