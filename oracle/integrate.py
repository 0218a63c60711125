"""Rigid-water drift, kicks, thermostats and pressure, float64 (oracle).

Restates, vectorised over molecules:
  integrate_rigid_water   src/solvent/opc_settle.rs:51-198
  kick_and_drift          src/integrate.rs:478-511
  kick_and_calc_accel     src/integrate.rs:515-562
  drift                   src/integrate.rs:566-587
  LangevinMiddle step     src/integrate.rs:100-212
  VerletVelocity + CSVR   src/integrate.rs:213-317
  measure_kinetic_energy(_translational)  src/thermostat.rs:46-84
  apply_thermostat_csvr   src/thermostat.rs:258-304
  apply_langevin_thermostat  src/thermostat.rs:308-362
  measure_pressure        src/barostat.rs:419-431
  Barostat::scale_factor, apply_isotropic  src/barostat.rs:329-413
  zero_linear_momentum    src/com_zero.rs:57-81
and the engine's deliberate deviations from them: the CSVR scale and the
temperature from the rigid-body kinetic energy (rigid_kinetic_energy), the
barostat driven by the molecular virial (intramolecular_virial).
Noise comes from oracle.philox (the engine's stream) instead of the
reference's unseeded ThreadRng.
"""
import numpy as np

from . import opc, philox

MAX_ACCEL = 1e5  # src/integrate.rs:26


def min_image(d, ext):
    return d - np.round(d / ext) * ext


def wrap(p, lo, ext):
    return lo + np.mod(p - lo, ext)


def rodrigues(r, omega, dt):
    """Rotate r by |omega| dt about omega (src/solvent/opc_settle.rs:51-67)."""
    od = omega * dt
    th = np.linalg.norm(od, axis=-1, keepdims=True)
    small = th < 1e-12
    ths = np.where(small, 1.0, th)
    n = od / ths
    c = np.cos(th)
    s = np.sin(th)
    rot = r * c + np.cross(n, r) * s + n * np.sum(n * r, axis=-1, keepdims=True) * (1.0 - c)
    wxr = np.cross(od, r)
    ser = r + wxr + np.cross(od, wxr) * 0.5
    return np.where(small, ser, rot)


def solve_sym3(ixx, iyy, izz, ixy, ixz, iyz, b):
    """I^-1 b by the adjugate (src/solvent/opc_settle.rs:69-95)."""
    det = (ixx * (iyy * izz - iyz * iyz) - ixy * (ixy * izz - iyz * ixz)
           + ixz * (ixy * iyz - iyy * ixz))
    ok = np.abs(det) >= 1e-12
    inv_det = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
    i00 = (iyy * izz - iyz * iyz) * inv_det
    i01 = (ixz * iyz - ixy * izz) * inv_det
    i02 = (ixy * iyz - ixz * iyy) * inv_det
    i11 = (ixx * izz - ixz * ixz) * inv_det
    i12 = (ixz * ixy - ixx * iyz) * inv_det
    i22 = (ixx * iyy - ixy * ixy) * inv_det
    bx, by, bz = b[:, 0], b[:, 1], b[:, 2]
    return np.stack([i00 * bx + i01 * by + i02 * bz,
                     i01 * bx + i11 * by + i12 * bz,
                     i02 * bx + i12 * by + i22 * bz], axis=1)


def rigid_water_drift(wpos, wvel, dt, lo, ext):
    """integrate_rigid_water for all molecules.

    wpos, wvel: (nw, 3, 3) arrays [O, H0, H1].  Returns new (wpos, wvel, m,
    constraint_virial).
    """
    mo, mh = float(opc.O_MASS), float(opc.H_MASS)
    mt = float(opc.MASS_WATER_MOL)
    o = wpos[:, 0]
    h0 = o + min_image(wpos[:, 1] - o, ext)
    h1 = o + min_image(wpos[:, 2] - o, ext)
    vo, vh0, vh1 = wvel[:, 0], wvel[:, 1], wvel[:, 2]
    r_com = (o * mo + h0 * mh + h1 * mh) / mt
    v_com = (vo * mo + vh0 * mh + vh1 * mh) / mt
    r_o, r_h0, r_h1 = o - r_com, h0 - r_com, h1 - r_com
    u_o, u_h0, u_h1 = vo - v_com, vh0 - v_com, vh1 - v_com
    L = np.cross(r_o, u_o) * mo + np.cross(r_h0, u_h0) * mh + np.cross(r_h1, u_h1) * mh

    def acc(r, m):
        x, y, z = r[:, 0], r[:, 1], r[:, 2]
        r2 = x * x + y * y + z * z
        return m * (r2 - x * x), m * (r2 - y * y), m * (r2 - z * z), -m * x * y, -m * x * z, -m * y * z

    terms = [acc(r_o, mo), acc(r_h0, mh), acc(r_h1, mh)]
    ixx, iyy, izz, ixy, ixz, iyz = (terms[0][k] + terms[1][k] + terms[2][k] for k in range(6))
    w = solve_sym3(ixx, iyy, izz, ixy, ixz, iyz, L)
    delta = v_com * dt
    r_o2 = rodrigues(r_o, w, dt)
    r_h02 = rodrigues(r_h0, w, dt)
    r_h12 = rodrigues(r_h1, w, dt)
    new_o = wrap(r_com + delta + r_o2, lo, ext)
    new_h0 = new_o + min_image(r_com + delta + r_h02 - new_o, ext)
    new_h1 = new_o + min_image(r_com + delta + r_h12 - new_o, ext)
    v_o2 = np.cross(w, r_o2)
    v_h02 = np.cross(w, r_h02)
    v_h12 = np.cross(w, r_h12)
    nv = np.stack([v_com + v_o2, v_com + v_h02, v_com + v_h12], axis=1)
    npos = np.stack([new_o, new_h0, new_h1], axis=1)
    bis = (new_h0 - new_o) + (new_h1 - new_o)
    m = new_o + bis / np.linalg.norm(bis, axis=1, keepdims=True) * float(opc.O_EP_R)
    dv_h0 = v_h02 - u_h0
    dv_h1 = v_h12 - u_h1
    vir = np.sum(np.sum((r_h02 - r_o2) * dv_h0 * (mh / dt), axis=1)
                 + np.sum((r_h12 - r_o2) * dv_h1 * (mh / dt), axis=1))
    return npos, nv, m, float(vir)


def kinetic_energy(state):
    """measure_kinetic_energy (src/thermostat.rs:46-64), kcal/mol."""
    ke = 0.0
    dyn = ~state["atom_static"]
    if len(state["atom_vel"]):
        v = state["atom_vel"][dyn]
        ke += float(np.sum(state["atom_mass"][dyn] * np.sum(v * v, axis=1)))
    wv = state["water_vel"]
    if len(wv):
        m = np.array([float(opc.O_MASS), float(opc.H_MASS), float(opc.H_MASS)])
        ke += float(np.sum(m[None, :] * np.sum(wv * wv, axis=2)))
    return ke * 0.5 / float(opc.KCAL_TO_NATIVE)


def kinetic_energy_translational(state):
    """measure_kinetic_energy_translational (src/thermostat.rs:69-84)."""
    ke = 0.0
    dyn = ~state["atom_static"]
    if len(state["atom_vel"]):
        v = state["atom_vel"][dyn]
        ke += float(np.sum(state["atom_mass"][dyn] * np.sum(v * v, axis=1)))
    wv = state["water_vel"]
    if len(wv):
        mo, mh, mt = float(opc.O_MASS), float(opc.H_MASS), float(opc.MASS_WATER_MOL)
        vc = (wv[:, 0] * mo + wv[:, 1] * mh + wv[:, 2] * mh) / mt
        ke += float(np.sum(mt * np.sum(vc * vc, axis=1)))
    return ke * 0.5 / float(opc.KCAL_TO_NATIVE)


def pressure_bar(ke_trans, virial_kcal, volume):
    """measure_pressure (src/barostat.rs:419-431)."""
    return (2.0 * ke_trans + virial_kcal) / (3.0 * volume) * opc.BAR_PER_KCAL_MOL_PER_ANSTROM_CUBED


def langevin_ou(state, dt, gamma, temp, step, seed):
    """apply_langevin_thermostat (src/thermostat.rs:308-362) with the engine's
    Philox stream: particle id = atom index for solute atoms, n_atoms +
    3*water + site for water sites (site 0 O, 1 H0, 2 H1)."""
    c = np.exp(-gamma * dt)
    s2 = max(1.0 - c * c, 0.0)
    num = float(opc.KB_A2_PS2_PER_K_PER_AMU) * temp * s2
    na = len(state["atom_vel"])
    nw = len(state["water_vel"])
    if na:
        dyn = ~state["atom_static"]
        xi = philox.ou_normals(np.arange(na, dtype=np.uint32), step, seed)
        sig = np.sqrt(num / np.where(dyn, state["atom_mass"], 1.0))
        newv = c * state["atom_vel"] + sig[:, None] * xi
        state["atom_vel"] = np.where(dyn[:, None], newv, state["atom_vel"])
    if nw:
        ids = (na + np.arange(3 * nw)).astype(np.uint32)
        xi = philox.ou_normals(ids, step, seed).reshape(nw, 3, 3)
        m = np.array([float(opc.O_MASS), float(opc.H_MASS), float(opc.H_MASS)])
        sig = np.sqrt(num / m)
        state["water_vel"] = c * state["water_vel"] + sig[None, :, None] * xi


def csvr(state, dt, tau, temp, dof, step, seed):
    """apply_thermostat_csvr (src/thermostat.rs:258-304); chi-square draw as
    2 * Gamma((dof-1)/2) from oracle.philox.gamma_marsaglia_tsang."""
    if tau <= 0.0:
        return
    dof = float(max(dof, 2))
    ke = kinetic_energy(state)
    if ke < 1e-20:
        return
    c = np.exp(-dt / tau)
    r = philox.csvr_normal(step, seed)
    chi = 2.0 * philox.gamma_marsaglia_tsang(0.5 * (dof - 1.0), step, seed)
    ke_t = 0.5 * dof * opc.GAS_CONST_R * temp
    kp = ke * c + ke_t * (1.0 - c) * ((chi + r * r) / dof) + 2.0 * r * np.sqrt(c * (1.0 - c) * ke * ke_t / dof)
    kp = max(kp, 1e-20)
    lam = np.sqrt(kp / ke)
    dyn = ~state["atom_static"]
    state["atom_vel"][dyn] *= lam
    state["water_vel"] *= lam


def zero_linear_momentum(state):
    """zero_linear_momentum (src/com_zero.rs:57-81)."""
    dyn = ~state["atom_static"]
    msum = float(np.sum(state["atom_mass"][dyn]))
    p = np.sum(state["atom_mass"][dyn, None] * state["atom_vel"][dyn], axis=0) if dyn.any() else np.zeros(3)
    nw = len(state["water_vel"])
    if nw:
        m = np.array([float(opc.O_MASS), float(opc.H_MASS), float(opc.H_MASS)])
        msum += float(opc.MASS_WATER_MOL) * nw
        p = p + np.sum(m[None, :, None] * state["water_vel"], axis=(0, 1))
    if msum <= 1e-6:
        return
    vc = p / msum
    state["atom_vel"][dyn] -= vc
    state["water_vel"] -= vc[None, None, :]


def _constraints(state):
    """(heavy, H, r0^2, inverse-mass sum) per constraint, heavy end first."""
    c = state.get("constraints")
    if c is None or len(c) == 0:
        return None
    c = np.asarray(c, np.int64).reshape(-1, 2)
    m = state["atom_mass"]
    heavy = np.where(m[c[:, 0]] >= m[c[:, 1]], c[:, 0], c[:, 1])
    hyd = np.where(heavy == c[:, 0], c[:, 1], c[:, 0])
    r02 = np.asarray(state["constraint_r0"], np.float64) ** 2
    return heavy, hyd, r02, 1.0 / m[heavy] + 1.0 / m[hyd]


def _in_unit_order(state):
    """Constraint indices grouped by heavy atom in atom order (the order in
    which each unit's constraints are applied)."""
    cs = _constraints(state)
    heavy = cs[0]
    return np.argsort(heavy, kind="stable")


def lincs_hydrogens(state, dt, order=4, iters=1):
    """lincs_hydrogens (src/bonded.rs:218-284): ``order`` projection passes
    along each bond, then ``iters`` SHAKE-style passes, sequentially over
    the constraints; returns the constraint virial estimate sum r_ij . f_i
    with f_i from the heavy atom's displacement (native units)."""
    cs = _constraints(state)
    if cs is None:
        return 0.0
    heavy, hyd, r02, im = cs
    x = state["atom_pos"]
    m = state["atom_mass"]
    fixed = state["atom_static"]
    x0 = x.copy()
    seq = _in_unit_order(state)
    for _ in range(order):
        for c in seq:
            i, j = heavy[c], hyd[c]
            d = x[j] - x[i]
            dl = max(np.linalg.norm(d), 1.1920929e-7)
            b = d / dl
            corr = b * ((np.sqrt(r02[c]) - b @ d) / im[c])
            if not fixed[i]:
                x[i] -= corr / m[i]
            if not fixed[j]:
                x[j] += corr / m[j]
    for _ in range(iters):
        for c in seq:
            i, j = heavy[c], hyd[c]
            d = x[j] - x[i]
            d2 = d @ d
            corr = d * ((d2 - r02[c]) / (2.0 * im[c] * max(d2, 1e-8)))
            if not fixed[i]:
                x[i] += corr / m[i]
            if not fixed[j]:
                x[j] -= corr / m[j]
    inv_dt2 = 1.0 / (dt * dt)
    w = 0.0
    for c in seq:
        i, j = heavy[c], hyd[c]
        w += float((x[j] - x[i]) @ ((x[i] - x0[i]) * (m[i] * inv_dt2)))
    return w


def shake_old_bonds(state, x_ref, dt, sweeps=32, tol=1e-6):
    """RATTLE's position stage (Andersen 1983): SHAKE iterations with the
    corrections along the bond vectors of ``x_ref`` (the positions at the
    start of the drift), per unit, until every |d|^2 is within ``tol`` of
    r0^2; returns the constraint virial estimate as lincs_hydrogens does."""
    cs = _constraints(state)
    if cs is None:
        return 0.0
    heavy, hyd, r02, im = cs
    x = state["atom_pos"]
    m = state["atom_mass"]
    fixed = state["atom_static"]
    x0 = x.copy()
    seq = _in_unit_order(state)
    for _ in range(sweeps):
        done = True
        for c in seq:
            i, j = heavy[c], hyd[c]
            d = x[j] - x[i]
            diff = d @ d - r02[c]
            if abs(diff) > tol * r02[c]:
                done = False
            ro = x_ref[j] - x_ref[i]
            corr = ro * (diff / (2.0 * im[c] * (d @ ro)))
            if not fixed[i]:
                x[i] += corr / m[i]
            if not fixed[j]:
                x[j] -= corr / m[j]
        if done:
            break
    inv_dt2 = 1.0 / (dt * dt)
    w = 0.0
    for c in range(len(heavy)):
        i, j = heavy[c], hyd[c]
        fi = (x[i] - x0[i]) * (m[i] * inv_dt2)
        w += (x[j] - x[i]) @ fi
    return w


def rattle_hydrogens_converged(state, sweeps=8):
    """The velocity projection repeated so that coupled bonds all hold."""
    for _ in range(sweeps):
        rattle_hydrogens(state)


def rattle_hydrogens(state):
    """rattle_hydrogens (src/bonded.rs:288-304)."""
    cs = _constraints(state)
    if cs is None:
        return
    heavy, hyd, _, im = cs
    x, vel, m = state["atom_pos"], state["atom_vel"], state["atom_mass"]
    for c in _in_unit_order(state):
        i, j = heavy[c], hyd[c]
        r = x[j] - x[i]
        corr = r * (((vel[j] - vel[i]) @ r) / (im[c] * max(r @ r, 1e-8)))
        vel[i] += corr / m[i]
        vel[j] -= corr / m[j]


def kick_and_calc_accel(state, forces, dt, rattle_velocities=False):
    """kick_and_calc_accel (src/integrate.rs:515-562), with RATTLE when the
    state carries constraints (iterated to convergence with
    ``rattle_velocities``).

    ``forces``: dict with f_atoms (na,3), f_water (nw,4,3) [O,H0,H1,M].
    """
    na = len(state["atom_vel"])
    if na:
        dyn = ~state["atom_static"]
        a = forces["f_atoms"] * (float(opc.KCAL_TO_NATIVE) / state["atom_mass"])[:, None]
        amag = np.linalg.norm(a, axis=1)
        big = amag * amag > MAX_ACCEL * MAX_ACCEL
        a = np.where(big[:, None], a / np.where(big, amag, 1.0)[:, None] * MAX_ACCEL, a)
        state["atom_accel"] = np.where(dyn[:, None], a, 0.0)
        state["atom_vel"] = state["atom_vel"] + state["atom_accel"] * dt
        if rattle_velocities:
            rattle_hydrogens_converged(state)
        else:
            rattle_hydrogens(state)
    fw = forces["f_water"]
    if len(fw):
        fo, fh0, fh1 = opc.project_ep_force(fw[:, 0], fw[:, 1], fw[:, 2], fw[:, 3])
        acc = np.stack([fo * float(opc.ACCEL_CONV_WATER_O), fh0 * float(opc.ACCEL_CONV_WATER_H),
                        fh1 * float(opc.ACCEL_CONV_WATER_H)], axis=1)
        state["water_accel"] = acc
        state["water_vel"] = state["water_vel"] + acc * dt


def kick_and_drift(state, dt_kick, dt_drift, lo, ext, rattle_velocities=False):
    """kick_and_drift (src/integrate.rs:478-511); with constraints,
    lincs_hydrogens(dt_kick) and RATTLE follow (:498-507).  With
    ``rattle_velocities``: RATTLE's position stage instead (shake_old_bonds,
    velocities following the displacement, v += dx / dt_drift), the engine's
    DYN_FLAG_RATTLE_VELOCITIES."""
    if len(state["atom_vel"]):
        dyn = ~state["atom_static"]
        x_ref = state["atom_pos"].copy()
        v = state["atom_vel"] + state["atom_accel"] * dt_kick
        state["atom_vel"] = np.where(dyn[:, None], v, state["atom_vel"])
        state["atom_pos"] = np.where(dyn[:, None], state["atom_pos"] + state["atom_vel"] * dt_drift,
                                     state["atom_pos"])
        if rattle_velocities:
            x_before = state["atom_pos"].copy()
            state["virial_constraints"] = shake_old_bonds(state, x_ref, dt_kick)
            dx = (state["atom_pos"] - x_before) / dt_drift
            state["atom_vel"] = np.where(dyn[:, None], state["atom_vel"] + dx, state["atom_vel"])
        else:
            state["virial_constraints"] = lincs_hydrogens(state, dt_kick)
            rattle_hydrogens(state)
    if len(state["water_vel"]):
        state["water_vel"] = state["water_vel"] + state["water_accel"] * dt_kick
        p, v, m, vir = rigid_water_drift(state["water_pos"], state["water_vel"], dt_drift, lo, ext)
        state["water_pos"], state["water_vel"], state["water_m"] = p, v, m
        return vir
    return 0.0


def drift(state, dt, lo, ext):
    """drift (src/integrate.rs:566-587) without H constraints."""
    if len(state["atom_vel"]):
        dyn = ~state["atom_static"]
        state["atom_pos"] = np.where(dyn[:, None], state["atom_pos"] + state["atom_vel"] * dt,
                                     state["atom_pos"])
    if len(state["water_vel"]):
        p, v, m, _ = rigid_water_drift(state["water_pos"], state["water_vel"], dt, lo, ext)
        state["water_pos"], state["water_vel"], state["water_m"] = p, v, m


def _rigid_frames(wpos, wvel, ext):
    """COM position and velocity, angular momentum L, inertia tensor and
    angular velocity omega = I^-1 L of each water (the quantities
    integrate_rigid_water computes first, src/solvent/opc_settle.rs:107-150),
    with the H sites min-imaged next to O."""
    mo, mh = float(opc.O_MASS), float(opc.H_MASS)
    mt = float(opc.MASS_WATER_MOL)
    o = wpos[:, 0]
    h0 = o + min_image(wpos[:, 1] - o, ext)
    h1 = o + min_image(wpos[:, 2] - o, ext)
    vo, vh0, vh1 = wvel[:, 0], wvel[:, 1], wvel[:, 2]
    r_com = (o * mo + h0 * mh + h1 * mh) / mt
    v_com = (vo * mo + vh0 * mh + vh1 * mh) / mt
    rs = (o - r_com, h0 - r_com, h1 - r_com)
    us = (vo - v_com, vh0 - v_com, vh1 - v_com)
    ms = (mo, mh, mh)
    L = sum(np.cross(r, u) * m for r, u, m in zip(rs, us, ms))
    t = [0.0] * 6
    for r, m in zip(rs, ms):
        x, y, z = r[:, 0], r[:, 1], r[:, 2]
        r2 = x * x + y * y + z * z
        for k, val in enumerate((m * (r2 - x * x), m * (r2 - y * y), m * (r2 - z * z),
                                 -m * x * y, -m * x * z, -m * y * z)):
            t[k] = t[k] + val
    omega = solve_sym3(*t, L)
    return r_com, v_com, L, omega


def rigid_kinetic_energy(state, ext):
    """Kinetic energy that survives the next rigid drift, kcal/mol: per water
    M v_com^2 / 2 + omega . L / 2, plus the solute atoms' KE.  The engine's
    thermostat and temperature use it instead of the site KE of
    measure_kinetic_energy (src/thermostat.rs:46-64), whose constrained
    components the rigid drift removes."""
    ke = 0.0
    dyn = ~state["atom_static"]
    if len(state["atom_vel"]):
        v = state["atom_vel"][dyn]
        ke += float(np.sum(state["atom_mass"][dyn] * np.sum(v * v, axis=1)))
    if len(state["water_vel"]):
        _, vc, L, w = _rigid_frames(state["water_pos"], state["water_vel"], ext)
        ke += float(np.sum(float(opc.MASS_WATER_MOL) * np.sum(vc * vc, axis=1) + np.sum(w * L, axis=1)))
    return ke * 0.5 / float(opc.KCAL_TO_NATIVE)


def csvr_lambda(ke, dt, tau, temp, dof, step, seed):
    """Velocity scale of the CSVR update (Bussi, Donadio, Parrinello, J. Chem.
    Phys. 126, 014101 (2007); apply_thermostat_csvr, src/thermostat.rs:258-304)
    for kinetic energy ``ke`` (kcal/mol), with the engine's Philox draws."""
    dof = float(max(dof, 2))
    if tau <= 0.0 or ke <= 1e-20:
        return 1.0
    c = np.exp(-dt / tau)
    r = philox.csvr_normal(step, seed)
    chi = 2.0 * philox.gamma_marsaglia_tsang(0.5 * (dof - 1.0), step, seed)
    ke_t = 0.5 * dof * opc.GAS_CONST_R * temp
    kp = ke * c + ke_t * (1.0 - c) * ((chi + r * r) / dof) + 2.0 * r * np.sqrt(c * (1.0 - c) * ke * ke_t / dof)
    return float(np.sqrt(max(kp, 1e-20) / ke))


def intramolecular_virial(state, f_water, ext):
    """sum over waters and their sites of (r_site - R_com) . F_site (kcal/mol),
    sites O, H0, H1, M; subtracted from the site virial it gives the
    molecular virial of rigid molecules."""
    if len(state["water_vel"]) == 0:
        return 0.0
    wp = state["water_pos"]
    o = wp[:, 0]
    r_com, _, _, _ = _rigid_frames(wp, state["water_vel"], ext)
    sites = [o, o + min_image(wp[:, 1] - o, ext), o + min_image(wp[:, 2] - o, ext),
             o + min_image(state["water_m"] - o, ext)]
    return float(sum(np.sum((s - r_com) * f_water[:, k], axis=1).sum() for k, s in enumerate(sites)))


def crescale_mu(pressure, dt, temp, p_target, tau, kappa, volume, step, seed):
    """Linear scale factor of the stochastic cell rescaling barostat
    (Bernetti & Bussi, J. Chem. Phys. 153, 114107 (2020); scale_factor,
    src/barostat.rs:329-354): d ln V = kappa / tau (P - P0) dt +
    sqrt(2 kappa kB T dt / (tau V)) xi, clamped to +-0.1, mu = e^{d ln V / 3}."""
    xi = philox.csvr_normal(step, seed, stream=philox.STREAM_BARO)
    det = kappa / tau * (pressure - p_target) * dt
    sig = np.sqrt(2.0 * kappa * opc.KB_BAR_A3_PER_K * temp * dt / (tau * volume))
    dl = min(max(det + sig * xi, -0.1), 0.1)
    return float(np.exp(dl / 3.0))


def crescale_apply(state, mu, lam, lo, ext):
    """apply_isotropic (src/barostat.rs:357-413, which the reference leaves
    disabled at :367-368) as the engine applies it together with the CSVR
    scale: water molecules moved with their COM (geometry kept), solute
    atoms scaled about the box centre, velocities scaled by lam / mu, the box
    scaled about its centre.  Returns the new (lo, ext)."""
    cen = lo + 0.5 * ext
    vs = lam / mu
    state["water_vel"] = state["water_vel"] * vs
    dyn = ~state["atom_static"]
    if len(state["atom_vel"]):
        state["atom_vel"] = np.where(dyn[:, None], state["atom_vel"] * vs, state["atom_vel"])
    if mu == 1.0:
        return lo, ext
    if len(state["water_vel"]):
        r_com, _, _, _ = _rigid_frames(state["water_pos"], state["water_vel"], ext)
        sh = (r_com - cen) * (mu - 1.0)
        state["water_pos"] = state["water_pos"] + sh[:, None, :]
        if "water_m" in state:
            state["water_m"] = state["water_m"] + sh
    if len(state["atom_vel"]):
        state["atom_pos"] = np.where(dyn[:, None], cen + (state["atom_pos"] - cen) * mu, state["atom_pos"])
    e = ext * mu
    return cen - 0.5 * e, e


def step_langevin_middle(state, forces_fn, dt, gamma, temp, step, seed, lo, ext):
    """One LangevinMiddle step (src/integrate.rs:100-212): kick dt/2 and
    drift dt/2, the OU step on every site velocity, drift dt/2, forces,
    kick dt/2.  ``forces_fn(state)`` returns the oracle force dict."""
    kick_and_drift(state, dt / 2, dt / 2, lo, ext)
    langevin_ou(state, dt, gamma, temp, step, seed)
    drift(state, dt / 2, lo, ext)
    f = forces_fn(state)
    kick_and_calc_accel(state, f, dt / 2)
    return f


def step_verlet_csvr(state, forces_fn, dt, tau, temp, dof, step, seed, lo, ext, baro=None):
    """One VerletVelocity step with CSVR (src/integrate.rs:213-317): kick
    dt/2 and drift dt, forces, kick dt/2, the CSVR scale from the rigid-body
    KE, and with ``baro`` = dict(p_target, tau, kappa) the C-rescale step
    driven by the molecular pressure.  Returns (forces, lam, mu, pressure,
    lo, ext)."""
    state["virial_constraints"] = 0.0
    kick_and_drift(state, dt / 2, dt, lo, ext)
    # bond-to-H constraint virial (native units); the rigid waters enter
    # through the molecular virial instead
    vir_c = state["virial_constraints"] / float(opc.KCAL_TO_NATIVE)
    f = forces_fn(state)
    kick_and_calc_accel(state, f, dt / 2)
    ke_r = rigid_kinetic_energy(state, ext)
    lam = csvr_lambda(ke_r, dt, tau, temp, dof, step, seed) if tau else 1.0
    ket = kinetic_energy_translational(state) * lam * lam
    vol = float(np.prod(ext))
    w = f["virial"] + vir_c - intramolecular_virial(state, f["f_water"], ext)
    p = pressure_bar(ket, w, vol)
    mu = 1.0
    if baro is not None:
        mu = crescale_mu(p, dt, temp, baro["p_target"], baro["tau"], baro["kappa"], vol, step, seed)
    lo, ext = crescale_apply(state, mu, lam, lo, ext)
    return f, lam, mu, p, lo, ext
