"""OPC rigid 4-site water: constants and geometry (oracle restatement).

Constants follow src/solvent/mod.rs:58-94 and src/solvent/opc_settle.rs:41,
src/lib.rs:196-201 and src/non_bonded.rs:55-63.  They are kept as float32
values exactly as the reference declares them (``f32`` consts), and exposed
as float64 for the FP64 oracle arithmetic.
"""
import numpy as np

f32 = np.float32

# src/non_bonded.rs:63
CHARGE_UNIT_SCALER = f32(18.2223)
# src/non_bonded.rs:55-56
SCALE_LJ_14 = f32(0.5)
SCALE_COUL_14 = f32(1.0) / f32(1.2)
# src/lib.rs:196,201
KCAL_TO_NATIVE = f32(418.4)
NATIVE_TO_KCAL = f32(1.0) / KCAL_TO_NATIVE
# src/solvent/mod.rs:58-60
O_MASS = f32(16.0)
H_MASS = f32(1.008)
MASS_WATER_MOL = O_MASS + f32(2.0) * H_MASS
# src/solvent/mod.rs:66-71
O_EP_R = f32(0.15939833)
O_H_R = f32(0.87243313)
H_O_H_THETA = f32(1.808161105066)
H_O_H_THETA_HALF = f32(0.5) * H_O_H_THETA
# src/solvent/mod.rs:74-79
SIGMA_FACTOR = f32(2.0) / f32(1.122462048309373)
O_RSTAR = f32(1.777167268)
O_SIGMA = O_RSTAR * SIGMA_FACTOR
O_EPS = f32(0.2128008130)
# src/solvent/mod.rs:82-83
Q_H = f32(0.6791) * CHARGE_UNIT_SCALER
Q_EP = f32(-2.0) * Q_H
# src/solvent/opc_settle.rs:41
RA = f32(0.5395199719801114)
# src/solvent/mod.rs:89-90
C_H = (O_EP_R / RA) / f32(2.0)
C_O = f32(1.0) - f32(2.0) * C_H
# src/solvent/mod.rs:93-94
ACCEL_CONV_WATER_O = KCAL_TO_NATIVE / O_MASS
ACCEL_CONV_WATER_H = KCAL_TO_NATIVE / H_MASS
# src/thermostat.rs:15,19
GAS_CONST_R = 0.0019872041
KB_A2_PS2_PER_K_PER_AMU = f32(0.83144626)
# src/barostat.rs:21,25
BAR_PER_KCAL_MOL_PER_ANSTROM_CUBED = 69476.95457055373
KB_BAR_A3_PER_K = 138.0649

# Site order used throughout the engine: O, H0, H1, M (the reference's
# WaterSite enum is O=1, M=2, H0=3, H1=4: src/solvent/mod.rs:256-261).
SITE_CHARGES = np.array([0.0, Q_H, Q_H, Q_EP], dtype=np.float64)


def quat_rotate(q, v):
    """Rotate vectors v (..., 3) by unit quaternions q (..., 4) = (w, x, y, z)."""
    w = q[..., 0:1]
    u = q[..., 1:4]
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def water_sites_from_orientation(o_pos, quat):
    """Positions of O, H0, H1, M for molecules at ``o_pos`` with orientations.

    Restates WaterMolOpc::new (src/solvent/mod.rs:337-353): the body z axis is
    the HOH bisector, the body x axis spans the molecular plane, H0/H1 sit at
    +/- half the HOH angle from the bisector at O_H_R, and M sits on the
    normalised bisector at O_EP_R.  Computed in float64, returned float32.
    """
    o = np.asarray(o_pos, dtype=np.float64)
    z_local = quat_rotate(quat, np.array([0.0, 0.0, 1.0]))
    e_local = quat_rotate(quat, np.array([1.0, 0.0, 0.0]))
    c = np.cos(float(H_O_H_THETA_HALF))
    s = np.sin(float(H_O_H_THETA_HALF))
    h0_dir = z_local * c + e_local * s
    h1_dir = z_local * c - e_local * s
    h0_dir /= np.linalg.norm(h0_dir, axis=-1, keepdims=True)
    h1_dir /= np.linalg.norm(h1_dir, axis=-1, keepdims=True)
    h0 = o + h0_dir * float(O_H_R)
    h1 = o + h1_dir * float(O_H_R)
    bis = (h0 - o) + (h1 - o)
    m = o + bis / np.linalg.norm(bis, axis=-1, keepdims=True) * float(O_EP_R)
    return (o.astype(np.float32), h0.astype(np.float32),
            h1.astype(np.float32), m.astype(np.float32))


def virtual_site(o, h0, h1):
    """M position on the HOH bisector (src/solvent/mod.rs:411-422), FP64."""
    bis = (h0 - o) + (h1 - o)
    return o + bis / np.linalg.norm(bis, axis=-1, keepdims=True) * float(O_EP_R)


def project_ep_force(f_o, f_h0, f_h1, f_m):
    """Move the M-site force onto O and H (src/solvent/mod.rs:397-406)."""
    return (f_o + f_m * float(C_O), f_h0 + f_m * float(C_H), f_h1 + f_m * float(C_H))
