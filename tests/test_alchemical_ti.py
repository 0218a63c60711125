"""Thermodynamic-integration helpers (dynamics_b200.alchemical) on
synthetic windows with a known integral."""
import numpy as np
import pytest

from dynamics_b200 import alchemical as al


def test_ti_of_a_linear_profile():
    lams = np.linspace(0.0, 1.0, 11)
    w = [al.LambdaWindow(float(l), 3.0 - 4.0 * l, 0.1) for l in lams]
    assert abs(al.free_energy_ti(w) - 1.0) < 1e-12  # integral of 3 - 4 l over [0, 1]
    est = al.free_energy_ti_with_sem(w)
    expect = np.sqrt(sum((0.5 * 0.1) ** 2 * (0.01 + 0.01) for _ in range(10)))
    assert abs(est.standard_error - expect) < 1e-12


def test_collect_window_from_frames():
    rng = np.random.default_rng(0)
    x = rng.normal(5.0, 2.0, 400)
    frames = [{"dh_dl": float(v)} for v in x] + [{"step": 1}]
    w = al.collect_window(0.3, frames)
    assert w.lam == 0.3 and abs(w.mean_dh_dl - x.mean()) < 1e-12
    assert abs(w.sem_dh_dl - x.std(ddof=1) / np.sqrt(len(x))) < 1e-12
    assert al.mean_coupled_interaction_kcal(frames) == pytest.approx(-x.mean())


def test_errors():
    with pytest.raises(al.AlchemicalError):
        al.free_energy_ti([al.LambdaWindow(0.0, 1.0, 0.0)])
    with pytest.raises(al.AlchemicalError):
        al.free_energy_ti([al.LambdaWindow(0.5, 1.0, 0.0), al.LambdaWindow(0.2, 1.0, 0.0)])
    with pytest.raises(al.AlchemicalError):
        al.collect_window(0.0, [{"step": 3}])
