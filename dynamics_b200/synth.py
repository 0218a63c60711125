"""Seeded synthetic systems of the benchmark shapes.

No public dataset is involved; systems are generated from the OPC geometry
(src/solvent/mod.rs:58-94) and, for peptides, from ff19SB residue data
extracted from the reference's parameter files (see
dynamics_b200/data/README).  The water generator restates the reference's
lattice-with-random-orientation idea (src/solvent/template_creation.rs:51-120)
and its rigid-body Maxwell-Boltzmann velocities (src/thermostat.rs:96-215).

Returned systems are plain dicts of numpy arrays (the layout documented in
dynamics_b200.md).
"""
import numpy as np

# OPC constants (float32 values of src/solvent/mod.rs:58-94)
O_MASS = np.float32(16.0)
H_MASS = np.float32(1.008)
O_EP_R = np.float32(0.15939833)
O_H_R = np.float32(0.87243313)
HOH = np.float32(1.808161105066)
CHARGE_UNIT_SCALER = np.float32(18.2223)
KB_NATIVE = 0.83144626          # amu A^2 ps^-2 / K
GAS_CONST_R = 0.0019872041      # kcal/mol/K
KCAL_TO_NATIVE = 418.4


def random_quaternions(rng, n):
    q = rng.normal(size=(n, 4))
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def _rotate(q, v):
    w = q[:, 0:1]
    u = q[:, 1:4]
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def water_geometry(o, quat):
    """H0, H1 positions for O at ``o`` with orientations ``quat``
    (WaterMolOpc::new, src/solvent/mod.rs:337-353), float64."""
    z = _rotate(quat, np.broadcast_to([0.0, 0.0, 1.0], o.shape))
    x = _rotate(quat, np.broadcast_to([1.0, 0.0, 0.0], o.shape))
    c, s = np.cos(float(HOH) / 2), np.sin(float(HOH) / 2)
    d0 = z * c + x * s
    d1 = z * c - x * s
    d0 /= np.linalg.norm(d0, axis=1, keepdims=True)
    d1 /= np.linalg.norm(d1, axis=1, keepdims=True)
    return o + d0 * float(O_H_R), o + d1 * float(O_H_R)


def lattice_sites(box_len, n_min):
    """A cubic lattice with at least n_min sites filling [0, L)^3."""
    k = int(np.ceil(n_min ** (1.0 / 3.0) - 1e-9))
    spacing = box_len / k
    g = (np.arange(k) + 0.5) * spacing
    xs, ys, zs = np.meshgrid(g, g, g, indexing="ij")
    return np.stack([xs.ravel(), ys.ravel(), zs.ravel()], axis=1), spacing


def _min_image(d, box_len):
    return d - np.round(d / box_len) * box_len


def orient_waters(o, box_len, rng, n_sweeps=30, min_hh=1.7, solute=None):
    """Random orientations, redrawn for molecules whose H sites sit closer
    than ``min_hh`` to another molecule's H (or to solute atoms)."""
    from scipy.spatial import cKDTree
    n = len(o)
    quat = random_quaternions(rng, n)
    for _ in range(n_sweeps):
        h0, h1 = water_geometry(o, quat)
        pts = np.concatenate([h0, h1], axis=0)
        mol = np.concatenate([np.arange(n), np.arange(n)])
        wrapped = np.mod(pts, box_len)
        tree = cKDTree(wrapped, boxsize=box_len)
        pairs = tree.query_pairs(min_hh, output_type="ndarray")
        bad = np.zeros(n, bool)
        if len(pairs):
            inter = mol[pairs[:, 0]] != mol[pairs[:, 1]]
            bad[mol[pairs[inter, 0]]] = True
        if solute is not None and len(solute):
            st = cKDTree(np.mod(solute, box_len), boxsize=box_len)
            d, _ = st.query(wrapped, k=1)
            bad[mol[d < 2.0]] = True
        if not bad.any():
            break
        quat[bad] = random_quaternions(rng, int(bad.sum()))
    return quat


def rigid_mb_velocities(wpos, temperature, rng):
    """Rigid-body Maxwell-Boltzmann velocities for waters
    (initialize_velocities, src/thermostat.rs:112-182): COM velocity from
    N(0, kT/M), angular momentum L ~ N(0, kT I), omega = I^-1 L."""
    n = len(wpos)
    m = np.array([float(O_MASS), float(H_MASS), float(H_MASS)])
    mt = m.sum()
    kt = KB_NATIVE * temperature
    com = np.einsum("k,nkd->nd", m, wpos) / mt
    r = wpos - com[:, None, :]
    inert = np.zeros((n, 3, 3))
    for k in range(3):
        rk = r[:, k]
        r2 = np.sum(rk * rk, axis=1)
        inert += m[k] * (r2[:, None, None] * np.eye(3)[None] - rk[:, :, None] * rk[:, None, :])
    w_eig, v_eig = np.linalg.eigh(inert)
    lp = rng.normal(size=(n, 3)) * np.sqrt(kt * np.maximum(w_eig, 0.0))
    L = np.einsum("nij,nj->ni", v_eig, lp)
    omega = np.linalg.solve(inert, L[:, :, None])[:, :, 0]
    vcom = rng.normal(size=(n, 3)) * np.sqrt(kt / mt)
    vel = vcom[:, None, :] + np.cross(omega[:, None, :], r)
    return vel


def remove_com_and_scale(sysd, temperature, dof):
    """Zero the total momentum and rescale to the exact temperature
    (src/thermostat.rs:191-214)."""
    m = np.array([float(O_MASS), float(H_MASS), float(H_MASS)])
    wv = sysd["water_vel"]
    p = np.einsum("k,nkd->d", m, wv)
    mtot = m.sum() * len(wv)
    av = sysd.get("atom_vel")
    am = sysd.get("atom_mass")
    if av is not None and len(av):
        p = p + np.sum(am[:, None] * av, axis=0)
        mtot += float(np.sum(am))
    vc = p / mtot
    wv -= vc
    ke = 0.5 * float(np.einsum("k,nkd,nkd->", m, wv, wv))
    if av is not None and len(av):
        av -= vc
        ke += 0.5 * float(np.sum(am[:, None] * av * av))
    ke_kcal = ke / KCAL_TO_NATIVE
    t_now = 2.0 * ke_kcal / (dof * GAS_CONST_R)
    lam = np.sqrt(temperature / t_now)
    wv *= lam
    if av is not None and len(av):
        av *= lam


def water_box(n_water, box_len, seed=0, temperature=300.0, sites=None, jitter=0.05):
    """``n_water`` OPC waters on a cubic lattice in a ``box_len`` cube with
    seeded orientations and rigid-body MB velocities at ``temperature``.

    Lattice sites get a small seeded jitter so that no O-O displacement sits
    exactly at half the box, where the periodic image is ambiguous."""
    rng = np.random.default_rng(seed)
    if sites is None:
        sites, _ = lattice_sites(box_len, n_water)
        if len(sites) > n_water:
            sites = sites[np.sort(rng.choice(len(sites), n_water, replace=False))]
    o = sites.astype(np.float64) + rng.uniform(-jitter, jitter, (len(sites), 3))
    o = np.mod(o, box_len)
    quat = orient_waters(o, box_len, rng)
    h0, h1 = water_geometry(o, quat)
    wpos = np.stack([o, h0, h1], axis=1)
    wvel = rigid_mb_velocities(wpos, temperature, rng)
    sysd = {
        "box_lo": np.zeros(3, np.float32),
        "box_hi": np.full(3, box_len, np.float32),
        "water_pos": wpos.astype(np.float32),
        "water_vel": wvel,
        "atom_pos": np.zeros((0, 3), np.float32),
        "atom_vel": np.zeros((0, 3), np.float32),
        "atom_mass": np.zeros(0, np.float32),
        "atom_q": np.zeros(0, np.float32),
        "atom_sigma": np.zeros(0, np.float32),
        "atom_eps": np.zeros(0, np.float32),
    }
    remove_com_and_scale(sysd, temperature, 6 * n_water - 3)
    sysd["water_vel"] = sysd["water_vel"].astype(np.float32)
    return sysd


def config1(seed=0):
    """512 OPC waters on an 8x8x8 lattice (3.1 A) in a 24.8 A cube, 300 K."""
    return water_box(512, 24.8, seed=seed)


def ewald_alpha(cutoff, rtol=1e-5):
    """alpha with erfc(alpha * cutoff) = rtol (GROMACS ewald-rtol rule)."""
    from scipy.special import erfcinv
    return float(erfcinv(rtol) / cutoff)


def fft_size(n):
    """Smallest m >= n whose prime factors are all in {2, 3, 5, 7}."""
    m = max(1, int(n))
    while True:
        k = m
        for p in (2, 3, 5, 7):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
        m += 1


def config4_sizes(n_sys=64, seed=0, lo=512, hi=8000):
    """Water counts drawn log-uniform from [lo, hi] (seeded)."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n_sys)).round().astype(int)


def batch_member(n_water, seed=0, density=0.0334, spacing=1.0):
    """One water box of the batched form: box sized to ``density`` waters per
    cubic angstrom and an FFT-friendly SPME grid of about ``spacing`` A.
    Returns (system, grid)."""
    box = float((n_water / density) ** (1.0 / 3.0))
    sysd = water_box(int(n_water), box, seed=seed)
    k = fft_size(int(np.ceil(box / spacing)))
    return sysd, (k, k, k)
