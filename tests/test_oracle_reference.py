"""The oracle against the reference's own known-answer tests.

The reference ships no golden vectors; its tests build every input inline.
Each test here restates one of them (file:line cited) with the same inputs
and tolerances, run against the oracle restatement, plus the published
Philox known-answer vectors and direct-sum checks of the SPME restatement.
"""
import numpy as np
import pytest

from oracle import bonded, integrate, opc, pairs, philox, spme

K_ELEC = float(opc.CHARGE_UNIT_SCALER) ** 2
SCALER = float(opc.CHARGE_UNIT_SCALER)


# ---------------------------------------------------------------- LJ ------
# src/tests/forces.rs:221-274
@pytest.mark.parametrize("r", [2.0, 2.5, 3.0, 4.5, 5.0, 7.0])
def test_lennard_jones_analytic(r):
    sigma, eps = 3.4, 0.086
    f, e = pairs.lj_force_energy(1.0 / r, sigma, eps)
    sr6 = (sigma / r) ** 6
    assert abs(f - 24 * eps * (2 * sr6 * sr6 - sr6) / r) <= 1e-4 * max(1.0, abs(f))
    assert abs(e - 4 * eps * (sr6 * sr6 - sr6)) <= 1e-4
    r_min = 2 ** (1 / 6) * sigma
    assert (f > 0) == (r < r_min)


def test_lennard_jones_minimum():
    sigma, eps = 3.4, 0.086
    _, e = pairs.lj_force_energy(1.0 / (2 ** (1 / 6) * sigma), sigma, eps)
    assert abs(e + eps) < 1e-4


# ------------------------------------------------ short-range Coulomb ------
# src/tests/forces.rs:377-423 (force = -dE/dr within 2 %)
@pytest.mark.parametrize("q1,q2", [(1.0, -1.0), (1.0, 1.0), (0.5, -0.3)])
@pytest.mark.parametrize("r", [3.0, 5.0, 8.0])
def test_coulomb_sr_force_energy_consistency(q1, q2, r):
    a, rc, h = 0.35, 10.0, 1e-3
    f, _ = pairs.coulomb_short_range(r, q1 * SCALER, q2 * SCALER, rc, a)
    _, ep = pairs.coulomb_short_range(r + h, q1 * SCALER, q2 * SCALER, rc, a)
    _, em = pairs.coulomb_short_range(r - h, q1 * SCALER, q2 * SCALER, rc, a)
    assert abs(f - (-(ep - em) / (2 * h))) <= 0.02 * abs(f)


# src/tests/forces.rs:427-462, 489-507
def test_coulomb_sr_sign_and_cutoff():
    a, rc = 0.35, 10.0
    for r in (3.0, 5.0, 8.0):
        f, e = pairs.coulomb_short_range(r, SCALER, SCALER, rc, a)
        assert f > 0 and e > 0
        f, e = pairs.coulomb_short_range(r, SCALER, -SCALER, rc, a)
        assert f < 0 and e < 0
    for r in (rc, rc + 0.5, rc + 2.0):
        f, e = pairs.coulomb_short_range(r, SCALER, -SCALER, rc, a)
        assert f == 0.0 and e == 0.0


# ------------------------------------------------------------- SPME ------
def _pair(dist, q1, q2, box=(50.0, 50.0, 50.0), alpha=0.35):
    box = np.asarray(box)
    c = box / 2
    r1 = c - np.array([dist / 2, 0, 0])
    r2 = c + np.array([dist / 2, 0, 0])
    q = np.array([q1, q2]) * SCALER
    grid = tuple(int(np.ceil(b)) for b in box)  # 1 A spacing, as the tests
    e_lr, f_lr, _ = spme.recip(np.stack([r1, r2]), q, np.zeros(3), box, grid, alpha)
    f_sr, e_sr = pairs.coulomb_short_range(dist, q[0], q[1], 10.0, alpha)
    # short-range force on charge 1 along dir = (r1 - r2)/|r1 - r2| = -x
    return f_lr[0, 0] - f_sr, e_sr + e_lr


# src/tests/spme.rs:147-168
@pytest.mark.parametrize("dist", [3.0, 5.0, 8.0])
def test_spme_energy_opposite_charges(dist):
    _, e = _pair(dist, 1.0, -1.0)
    assert abs((e - (-K_ELEC / dist)) / (-K_ELEC / dist)) < 0.01


# src/tests/spme.rs:171-187
@pytest.mark.parametrize("q", [0.5, 0.25])
def test_spme_energy_fractional_charges(q):
    _, e = _pair(5.0, q, -q)
    ev = -K_ELEC * q * q / 5.0
    assert abs((e - ev) / ev) < 0.01


# src/tests/spme.rs:225-270 (1 %, 2 % at 8 A)
@pytest.mark.parametrize("dist", [3.0, 5.0, 8.0])
def test_spme_force_magnitude(dist):
    fx, _ = _pair(dist, 1.0, -1.0)
    fv = K_ELEC / dist ** 2
    tol = 0.02 if dist >= 7 else 0.01
    assert abs((fx - fv) / fv) < tol


# src/tests/spme.rs:348-381
def test_spme_energy_non_cubic_box():
    _, e = _pair(5.0, 1.0, -1.0, box=(60.0, 30.0, 30.0))
    ev = -K_ELEC / 5.0
    assert abs((e - ev) / ev) < 0.01


# src/tests/spme.rs:396-440
@pytest.mark.parametrize("dist", [3.0, 5.0, 8.0])
def test_spme_force_like_charges(dist):
    fx, _ = _pair(dist, 1.0, 1.0)
    fv = -K_ELEC / dist ** 2
    tol = 0.02 if dist >= 7 else 0.01
    assert abs((fx - fv) / fv) < tol


# src/tests/spme.rs:454-491
@pytest.mark.parametrize("dist", [3.0, 5.0, 8.0])
def test_spme_force_matches_energy_gradient(dist):
    h = 0.01
    fx, _ = _pair(dist, 1.0, -1.0)
    _, ep = _pair(dist - h, 1.0, -1.0)  # r1 moved +h along x: distance shrinks by h
    _, em = _pair(dist + h, 1.0, -1.0)
    fnum = -(ep - em) / (2 * h)
    assert abs((fx - fnum) / fnum) < 0.02


def test_spme_matches_direct_ewald_sum():
    rng = np.random.default_rng(1)
    n = 40
    box = np.array([20.0, 22.0, 18.0])
    p = rng.uniform(0, 1, (n, 3)) * box
    q = rng.normal(size=n)
    q = (q - q.mean()) * SCALER
    e1, f1, _ = spme.recip(p, q, np.zeros(3), box, (32, 32, 32), 0.35, include_self=False)
    e2, f2 = spme.direct_recip(p, q, box, 0.35, kmax=14)
    assert abs(e1 - e2) / abs(e2) < 2e-4
    assert np.sqrt(np.sum((f1 - f2) ** 2) / np.sum(f2 ** 2)) < 2e-3


def test_spme_virial_is_minus_scaling_derivative():
    rng = np.random.default_rng(2)
    n = 30
    box = np.array([20.0, 20.0, 24.0])
    p = rng.uniform(0, 1, (n, 3)) * box
    q = rng.normal(size=n)
    q = (q - q.mean()) * SCALER
    _, _, w = spme.recip(p, q, np.zeros(3), box, (24, 24, 30), 0.3, include_self=False)

    def e(s):
        return spme.recip(p * s, q, np.zeros(3), box * s, (24, 24, 30), 0.3, include_self=False)[0]

    h = 1e-5
    assert abs(w - (-(e(1 + h) - e(1 - h)) / (2 * h))) < 1e-6 * max(1.0, abs(w))


def test_exclusion_correction_gradient():
    d = np.array([[0.9, 0.3, -0.2]])
    e0, f, _ = spme.exclusion_correction(d, np.zeros((1, 3)), [12.0], [-24.0], np.full(3, 50.0), 0.31)
    h = 1e-6
    for k in range(3):
        dp = d.copy(); dp[0, k] += h
        dm = d.copy(); dm[0, k] -= h
        ep = spme.exclusion_correction(dp, np.zeros((1, 3)), [12.0], [-24.0], np.full(3, 50.0), 0.31)[0]
        em = spme.exclusion_correction(dm, np.zeros((1, 3)), [12.0], [-24.0], np.full(3, 50.0), 0.31)[0]
        assert abs(f[0, k] + (ep - em) / (2 * h)) < 1e-5


# ----------------------------------------------------------- bonded ------
# src/tests/force_components.rs:67-110
@pytest.mark.parametrize("r", [1.2, 1.5, 1.8])
def test_bond_force_energy_matches_amber_harmonic(r):
    pos = np.array([[5.0, 5.0, 5.0], [5.0 + r, 5.0, 5.0]])
    f0, f1, e, _ = bonded.bonds(pos, np.array([[0, 1]]), np.array([120.0]), np.array([1.5]), np.full(3, 20.0))
    dr = r - 1.5
    assert abs(f0[0, 0] - 2 * 120 * dr) < 1e-5
    assert abs(e[0] - 120 * dr * dr) < 3e-5


def test_bond_force_uses_minimum_image():
    pos = np.array([[0.2, 5.0, 5.0], [9.0, 5.0, 5.0]])
    f0, _, e, _ = bonded.bonds(pos, np.array([[0, 1]]), np.array([100.0]), np.array([1.0]), np.full(3, 10.0))
    assert abs(f0[0, 0] + 40.0) < 1e-4
    assert abs(e[0] - 4.0) < 1e-4


def _fd_check(fn, pos, idx, *par, tol=1e-4):
    ext = np.full(3, 60.0)
    out = fn(pos, idx, *par, ext)
    forces = out[0] if isinstance(out[0], list) else out[:len(idx[0])]
    h = 1e-6
    for a in range(idx.shape[1]):
        for k in range(3):
            pp = pos.copy(); pp[idx[0, a], k] += h
            pm = pos.copy(); pm[idx[0, a], k] -= h
            ep = np.sum(fn(pp, idx, *par, ext)[-2])
            em = np.sum(fn(pm, idx, *par, ext)[-2])
            assert abs(forces[a][0, k] + (ep - em) / (2 * h)) < tol


# src/tests/force_components.rs:112-197 (finite-difference checks)
def test_angle_and_dihedral_gradients():
    rng = np.random.default_rng(3)
    pos = rng.normal(size=(4, 3)) * 1.3
    _fd_check(bonded.angles, pos[:3], np.array([[0, 1, 2]]), np.array([55.0]), np.array([1.9]))
    f, e, w = bonded.dihedrals(pos, np.array([[0, 1, 2, 3]]), np.array([1.3]), np.array([3.0]),
                               np.array([0.4]), np.full(3, 60.0))
    h = 1e-6
    for a in range(4):
        for k in range(3):
            pp = pos.copy(); pp[a, k] += h
            pm = pos.copy(); pm[a, k] -= h
            ep = bonded.dihedrals(pp, np.array([[0, 1, 2, 3]]), np.array([1.3]), np.array([3.0]),
                                  np.array([0.4]), np.full(3, 60.0))[1][0]
            em = bonded.dihedrals(pm, np.array([[0, 1, 2, 3]]), np.array([1.3]), np.array([3.0]),
                                  np.array([0.4]), np.full(3, 60.0))[1][0]
            assert abs(f[a][0, k] + (ep - em) / (2 * h)) < 1e-5


# ------------------------------------------------ KE / T / P ------
def _state(atom_mass=(), atom_vel=(), water_vel=None, static=()):
    na = len(atom_mass)
    return {
        "atom_mass": np.asarray(atom_mass, float), "atom_vel": np.asarray(atom_vel, float).reshape(na, 3),
        "atom_static": np.asarray(static if len(static) else [False] * na, bool),
        "water_vel": np.zeros((0, 3, 3)) if water_vel is None else np.asarray(water_vel, float),
    }


# src/tests/therm_baro.rs:26-44
def test_kinetic_energy_atoms():
    s = _state([12.0, 1.0], [[3, 0, 0], [0, 2, 0]])
    assert abs(integrate.kinetic_energy(s) - 0.5 * (108 + 4) / 418.4) < 1e-6 * 0.13


# src/tests/therm_baro.rs:46-66
def test_kinetic_energy_excludes_static():
    s = _state([12.0, 12.0], [[1, 0, 0], [10, 10, 10]], static=[False, True])
    assert abs(integrate.kinetic_energy(s) - 0.5 * 12 / 418.4) < 1e-9


# src/tests/therm_baro.rs:68-98
def test_kinetic_energy_includes_water():
    wv = np.array([[[2.0, 0, 0], [0, 1.0, 0], [0, 1.0, 0]]])
    s = _state(water_vel=wv)
    exp = 0.5 * (16 * 4 + 1.008 + 1.008) / 418.4
    assert abs(integrate.kinetic_energy(s) - exp) / exp < 1e-5


# src/tests/therm_baro.rs:100-166
def test_translational_kinetic_energy():
    wv = np.array([[[3.0, 0, 0]] * 3])
    s = _state(water_vel=wv)
    exp = 0.5 * float(opc.MASS_WATER_MOL) * 9 / 418.4
    assert abs(integrate.kinetic_energy_translational(s) - exp) / exp < 1e-5
    vh = 1.0
    vo = -2 * 1.008 / 16.0
    s = _state(water_vel=np.array([[[0, vo, 0], [0, vh, 0], [0, vh, 0]]]))
    assert integrate.kinetic_energy_translational(s) < 1e-5 * integrate.kinetic_energy(s)


# src/tests/therm_baro.rs:187-292 (ideal-gas pressure)
def test_pressure_ideal_gas():
    ke = 1.234
    vol = 60.0 ** 3
    p = integrate.pressure_bar(ke, 0.0, vol)
    assert abs(p - 2 * ke / (3 * vol) * opc.BAR_PER_KCAL_MOL_PER_ANSTROM_CUBED) < 1e-12


# --------------------------------------------------------- rigid water ------
def test_rigid_drift_preserves_geometry_and_momentum():
    from dynamics_b200 import synth
    s = synth.water_box(27, 9.3, seed=5)
    wp = s["water_pos"].astype(np.float64)
    wv = s["water_vel"].astype(np.float64)
    ext = np.full(3, 9.3)
    p2, v2, m2, _ = integrate.rigid_water_drift(wp, wv, 0.002, np.zeros(3), ext)
    for a, b in ((0, 1), (0, 2), (1, 2)):
        d0 = np.linalg.norm(integrate.min_image(wp[:, a] - wp[:, b], ext), axis=1)
        d1 = np.linalg.norm(integrate.min_image(p2[:, a] - p2[:, b], ext), axis=1)
        assert np.max(np.abs(d0 - d1)) < 1e-9
    # momentum is conserved up to the float32 molecular-mass constant the
    # reference normalises the COM with (src/solvent/mod.rs:60)
    mass = np.array([float(opc.O_MASS), float(opc.H_MASS), float(opc.H_MASS)])
    p0 = np.einsum("k,nkd->nd", mass, wv)
    p1 = np.einsum("k,nkd->nd", mass, v2)
    assert np.max(np.abs(p0 - p1)) < 1e-5 * np.max(np.abs(p0)) + 1e-3


# --------------------------------------------------------- Philox KAT ------
# Published known-answer vectors for Philox4x32-10 (Random123 kat_vectors)
@pytest.mark.parametrize("ctr,key,exp", [
    ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
])
def test_philox_known_answers(ctr, key, exp):
    out = philox.philox4x32(*[np.uint32(c) for c in ctr], *[np.uint32(k) for k in key])
    assert tuple(int(o) for o in out) == exp


def test_philox_normals_statistics():
    z = philox.ou_normals(np.arange(200000, dtype=np.uint32), 7, 1234)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1) < 0.01
