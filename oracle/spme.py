"""Smooth particle-mesh Ewald, float64 (oracle).

The reference delegates the reciprocal sum to the external crate
``ewald`` ^0.1.15 (Cargo.toml:42; call sites src/non_bonded.rs:681-875,
src/tests/spme.rs:46-117), whose source is not in the reference tree.  This
module restates the published method it implements -- Essmann et al.,
J. Chem. Phys. 103, 8577 (1995), cardinal B-splines of order 4 -- with the
reference's conventions at those call sites:

* charges are already scaled by sqrt(332.0522) (src/non_bonded.rs:58-63),
  so no Coulomb constant appears;
* positions are wrapped into the primary box before spreading
  (pack_pme_pos_q, src/non_bonded.rs:800-826);
* the returned reciprocal energy includes the Ewald self term
  -alpha/sqrt(pi) * sum q^2 (the reference's own test
  src/tests/spme.rs:147-168 only passes with it);
* the virial is the k-space trace sum_m E(m) (1 - 2 pi^2 |m|^2 / alpha^2)
  (forces_and_virial, src/non_bonded.rs:693).

A direct (non-mesh) Ewald reciprocal sum is provided to validate the mesh
restatement on small systems.
"""
import numpy as np
from scipy.special import erf

ORDER = 4


def bspline4(w):
    """Order-4 cardinal B-spline weights and derivatives.

    For fractional offset w in [0, 1) returns (theta, dtheta), each (..., 4),
    where theta[..., j] = M4(w + 3 - j) is the weight of grid point
    floor(u) - 3 + j, j = 0..3 (points in ascending order).
    """
    w = np.asarray(w, dtype=np.float64)
    w2 = w * w
    w3 = w2 * w
    one_m = 1.0 - w
    th = np.stack([
        one_m ** 3 / 6.0,                               # M4(w + 3), point b-3
        (3.0 * w3 - 6.0 * w2 + 4.0) / 6.0,              # M4(w + 2), point b-2
        (-3.0 * w3 + 3.0 * w2 + 3.0 * w + 1.0) / 6.0,   # M4(w + 1), point b-1
        w3 / 6.0,                                       # M4(w),     point b
    ], axis=-1)
    # d/du of M4(u - k) = M4'(w + 3 - j)
    dth = np.stack([
        -0.5 * one_m ** 2,
        1.5 * w2 - 2.0 * w,
        -1.5 * w2 + w + 0.5,
        0.5 * w2,
    ], axis=-1)
    return th, dth


def bspline_moduli(k, order=ORDER):
    """|b(m)|^2 for m = 0..k-1 (Essmann eq. 4.4 with M4(1,2,3) = 1/6, 4/6, 1/6)."""
    mvals = {1: 1.0 / 6.0, 2: 4.0 / 6.0, 3: 1.0 / 6.0}
    m = np.arange(k)
    den = np.zeros(k, dtype=np.complex128)
    for j in range(order - 1):
        den += mvals[j + 1] * np.exp(2j * np.pi * m * j / k)
    return 1.0 / np.abs(den) ** 2


def influence(grid, box_ext, alpha):
    """B(m) C(m) on the full grid (zero at m = 0) and the |m|^2 array."""
    k1, k2, k3 = grid
    lx, ly, lz = (float(v) for v in box_ext)
    vol = lx * ly * lz

    def mfreq(k, l):
        m = np.fft.fftfreq(k) * k  # 0,1,..,k/2-1,-k/2,..,-1
        return m / l

    mx = mfreq(k1, lx)[:, None, None]
    my = mfreq(k2, ly)[None, :, None]
    mz = mfreq(k3, lz)[None, None, :]
    m2 = mx * mx + my * my + mz * mz
    b = (bspline_moduli(k1)[:, None, None] * bspline_moduli(k2)[None, :, None]
         * bspline_moduli(k3)[None, None, :])
    with np.errstate(divide="ignore", invalid="ignore"):
        c = np.exp(-np.pi ** 2 * m2 / alpha ** 2) / (np.pi * vol * m2)
    c[0, 0, 0] = 0.0
    return b * c, m2


def fractional(pos, box_lo, box_ext, grid):
    """u = K (x - lo) / L for positions already wrapped into the box."""
    p = np.asarray(pos, dtype=np.float64)
    lo = np.asarray(box_lo, dtype=np.float64)
    ext = np.asarray(box_ext, dtype=np.float64)
    u = (p - lo) / ext * np.asarray(grid, dtype=np.float64)
    k = np.asarray(grid)
    u = np.mod(u, k)  # guard points exactly on the upper face
    return u


def spread(u, q, grid):
    """Charge grid Q (Essmann eq. 4.6) and the per-particle spline data."""
    k = np.asarray(grid)
    base = np.floor(u).astype(np.int64)
    w = u - base
    th, dth = bspline4(w)
    idx = (base[..., None] - 3 + np.arange(4)) % k[None, :, None]  # (n, 3, 4)
    qgrid = np.zeros(tuple(k), dtype=np.float64)
    for a in range(4):
        for b in range(4):
            wab = q * th[:, 0, a] * th[:, 1, b]
            for c in range(4):
                np.add.at(qgrid, (idx[:, 0, a], idx[:, 1, b], idx[:, 2, c]), wab * th[:, 2, c])
    return qgrid, idx, th, dth


def recip(pos, q, box_lo, box_ext, grid, alpha, include_self=True):
    """SPME reciprocal energy, forces and virial in float64.

    Returns (energy, forces (n, 3), virial).  ``energy`` includes the self
    term when ``include_self``.
    """
    q = np.asarray(q, dtype=np.float64)
    grid = tuple(int(g) for g in grid)
    u = fractional(pos, box_lo, box_ext, grid)
    qgrid, idx, th, dth = spread(u, q, grid)
    g, m2 = influence(grid, box_ext, alpha)
    fq = np.fft.fftn(qgrid)
    e_m = 0.5 * g * np.abs(fq) ** 2
    energy = float(np.sum(e_m))
    virial = float(np.sum(e_m * (1.0 - 2.0 * np.pi ** 2 * m2 / alpha ** 2)))
    phi = np.real(np.fft.ifftn(g * fq)) * qgrid.size
    n = len(q)
    f = np.zeros((n, 3))
    ext = np.asarray(box_ext, dtype=np.float64)
    kk = np.asarray(grid, dtype=np.float64)
    for a in range(4):
        for b in range(4):
            for c in range(4):
                ph = phi[idx[:, 0, a], idx[:, 1, b], idx[:, 2, c]]
                f[:, 0] += dth[:, 0, a] * th[:, 1, b] * th[:, 2, c] * ph
                f[:, 1] += th[:, 0, a] * dth[:, 1, b] * th[:, 2, c] * ph
                f[:, 2] += th[:, 0, a] * th[:, 1, b] * dth[:, 2, c] * ph
    f *= -(q[:, None] * kk[None, :] / ext[None, :])
    if include_self:
        energy += self_energy(q, alpha)
    return energy, f, virial


def self_energy(q, alpha):
    """Ewald self term -alpha/sqrt(pi) sum q^2."""
    q = np.asarray(q, dtype=np.float64)
    return float(-alpha / np.sqrt(np.pi) * np.sum(q * q))


def direct_recip(pos, q, box_ext, alpha, kmax):
    """Exact Ewald reciprocal sum (no mesh): energy and forces.

    E = 1/(2 pi V) sum_{m != 0} exp(-pi^2 m^2/alpha^2)/m^2 |S(m)|^2,
    m = (n1/Lx, n2/Ly, n3/Lz), |n_a| <= kmax.  Excludes the self term.
    """
    p = np.asarray(pos, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    ext = np.asarray(box_ext, dtype=np.float64)
    vol = float(np.prod(ext))
    rng = np.arange(-kmax, kmax + 1)
    n1, n2, n3 = np.meshgrid(rng, rng, rng, indexing="ij")
    nvec = np.stack([n1.ravel(), n2.ravel(), n3.ravel()], axis=1)
    nvec = nvec[np.any(nvec != 0, axis=1)]
    m = nvec / ext[None, :]
    m2 = np.sum(m * m, axis=1)
    coef = np.exp(-np.pi ** 2 * m2 / alpha ** 2) / m2 / (2.0 * np.pi * vol)
    phase = 2.0 * np.pi * (p @ m.T)  # (n, M)
    cs = np.cos(phase)
    sn = np.sin(phase)
    s_re = q @ cs
    s_im = q @ sn
    energy = float(np.sum(coef * (s_re ** 2 + s_im ** 2)))
    # dE/dr_i = coef * 2 * q_i * 2 pi m * (-sin(phase_i) S_re + cos(phase_i) S_im)
    g = (-sn * s_re[None, :] + cs * s_im[None, :]) * (coef * 4.0 * np.pi)[None, :]
    f = -(q[:, None] * (g @ m))
    return energy, f


def exclusion_correction(pos_i, pos_j, qi, qj, box_ext, alpha, scale=1.0):
    """Remove ``scale`` * qi qj erf(alpha r)/r for excluded pairs (float64).

    Returns (energy, force on i (n,3), virial).  Force on j is the negative.
    """
    d = np.asarray(pos_i, dtype=np.float64) - np.asarray(pos_j, dtype=np.float64)
    ext = np.asarray(box_ext, dtype=np.float64)
    d = d - np.round(d / ext) * ext
    r = np.sqrt(np.sum(d * d, axis=1))
    qq = np.asarray(qi, dtype=np.float64) * np.asarray(qj, dtype=np.float64) * scale
    ar = alpha * r
    e = -qq * erf(ar) / r
    # U = -qq erf(ar)/r;  F_i = -dU/dr * d/r
    du = qq * (erf(ar) / r ** 2 - 2.0 * alpha / np.sqrt(np.pi) * np.exp(-ar * ar) / r)
    fmag = -du
    f = d * (fmag / r)[:, None]
    return float(np.sum(e)), f, float(np.sum(fmag * r))
