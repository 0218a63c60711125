"""Trajectory files from snapshot frames (MdState.read_snapshots): CHARMM /
NAMD DCD and GROMACS TRR, the formats the reference writes through its
bio_files dependency (src/snapshot.rs:836-904).  XTC (compressed
coordinates) is not written.

A frame is a dict as read_snapshots returns it: ``pos`` (n, 3) in
angstrom (atoms, then O, H0, H1 of each water), optionally ``vel`` (A/ps)
and ``force`` (kcal/mol/A, all n sites), ``step``, ``time_ps``,
``box_lo`` / ``box_hi`` (A).

DCD: little-endian Fortran records (4-byte length before and after each):
an 84-byte header ("CORD" + 20 int32: frame count, first step, steps
between frames, total steps, five zeros, the time step as float32 bits,
unit-cell flag 1, zeros, version 24), a title record, the atom count, then
per frame a 48-byte unit cell (A, gamma, B, beta, alpha, C; angles in
degrees) and the X, Y and Z records of float32.

TRR: XDR (big-endian) frames, each a header (magic 1993, the version
string "GMX_trn_file", the byte sizes of the blocks that follow, atom
count, step, energy count, time and lambda) followed by the box (3 x 3), x,
v and f in nm, nm/ps and kJ/mol/nm, single precision.
"""
import struct

import numpy as np

KCAL_TO_KJ = 4.184
A_TO_NM = 0.1
# AKMA time unit (the DCD time step field) in ps
AKMA_PS = 4.888821e-2


def _rec(f, payload):
    f.write(struct.pack("<i", len(payload)))
    f.write(payload)
    f.write(struct.pack("<i", len(payload)))


def write_dcd(path, frames, steps_between=1, dt_ps=0.002, title="dynamics_b200 snapshots"):
    """Writes frames to a new DCD file at ``path``."""
    frames = list(frames)
    n = frames[0]["pos"].shape[0] if frames else 0
    first = int(frames[0]["step"]) if frames else 0
    icntrl = [0] * 20
    icntrl[0] = len(frames)
    icntrl[1] = first
    icntrl[2] = int(steps_between)
    icntrl[3] = int(steps_between) * len(frames)
    icntrl[10] = 1  # unit cell present
    icntrl[19] = 24
    head = b"CORD" + struct.pack("<9i", *icntrl[:9]) + struct.pack("<f", dt_ps / AKMA_PS) \
        + struct.pack("<10i", *icntrl[10:])
    line = title.encode()[:80].ljust(80)
    with open(path, "wb") as f:
        _rec(f, head)
        _rec(f, struct.pack("<i", 1) + line)
        _rec(f, struct.pack("<i", n))
        for fr in frames:
            lo = np.asarray(fr.get("box_lo", (0.0, 0.0, 0.0)), np.float64)
            hi = np.asarray(fr.get("box_hi", (0.0, 0.0, 0.0)), np.float64)
            a, b, c = hi - lo
            _rec(f, struct.pack("<6d", a, 90.0, b, 90.0, 90.0, c))
            p = np.asarray(fr["pos"], np.float32)
            for k in range(3):
                _rec(f, np.ascontiguousarray(p[:, k]).astype("<f4").tobytes())


def read_dcd(path):
    """(positions (frames, n, 3) float32, unit cells (frames, 6), header
    ints) of a DCD file written by write_dcd."""
    data = open(path, "rb").read()
    off = 0

    def rec():
        nonlocal off
        (ln,) = struct.unpack_from("<i", data, off)
        payload = data[off + 4: off + 4 + ln]
        (ln2,) = struct.unpack_from("<i", data, off + 4 + ln)
        if ln2 != ln:
            raise ValueError("corrupt DCD record")
        off += ln + 8
        return payload

    head = rec()
    if head[:4] != b"CORD":
        raise ValueError("not a DCD file")
    icntrl = list(struct.unpack_from("<20i", head, 4))
    rec()  # title
    (n,) = struct.unpack("<i", rec())
    pos, cells = [], []
    for _ in range(icntrl[0]):
        cells.append(struct.unpack("<6d", rec()) if icntrl[10] else (0.0,) * 6)
        xyz = [np.frombuffer(rec(), "<f4") for _ in range(3)]
        pos.append(np.stack(xyz, axis=1))
    return np.array(pos, np.float32).reshape(len(pos), n, 3), np.array(cells), icntrl


def _trr_frame(fr):
    p = np.asarray(fr["pos"], np.float64)
    n = p.shape[0]
    lo = np.asarray(fr.get("box_lo", (0.0, 0.0, 0.0)), np.float64)
    hi = np.asarray(fr.get("box_hi", (0.0, 0.0, 0.0)), np.float64)
    box = np.diag((hi - lo) * A_TO_NM)
    v = fr.get("vel")
    f = fr.get("force")
    if f is not None and np.asarray(f).shape[0] != n:
        f = None  # forces of some sites only: not written
    real = 4
    sizes = dict(ir=0, e=0, box=9 * real, vir=0, pres=0, top=0, sym=0, x=3 * n * real,
                 v=3 * n * real if v is not None else 0, f=3 * n * real if f is not None else 0)
    out = bytearray()
    out += struct.pack(">ii", 1993, 13)
    out += struct.pack(">i", 12) + b"GMX_trn_file"
    out += struct.pack(">13i", sizes["ir"], sizes["e"], sizes["box"], sizes["vir"], sizes["pres"],
                       sizes["top"], sizes["sym"], sizes["x"], sizes["v"], sizes["f"], n,
                       int(fr.get("step", 0)), 0)
    out += struct.pack(">ff", float(fr.get("time_ps", 0.0)), 0.0)
    out += box.astype(">f4").tobytes()
    out += (p * A_TO_NM).astype(">f4").tobytes()
    if v is not None:
        out += (np.asarray(v, np.float64) * A_TO_NM).astype(">f4").tobytes()
    if f is not None:
        out += (np.asarray(f, np.float64) * (KCAL_TO_KJ / A_TO_NM)).astype(">f4").tobytes()
    return bytes(out)


def write_trr(path, frames, append=False):
    """Writes (or appends) frames to a TRR file at ``path``."""
    with open(path, "ab" if append else "wb") as f:
        for fr in frames:
            f.write(_trr_frame(fr))


def read_trr(path):
    """Frames of a single-precision TRR file: dicts with step, time_ps,
    box (3, 3) nm, x (n, 3) nm, and v / f when present."""
    data = open(path, "rb").read()
    off = 0
    frames = []
    while off < len(data):
        magic, slen, ln = struct.unpack_from(">iii", data, off)
        if magic != 1993 or slen != 13 or ln != 12 or data[off + 12: off + 24] != b"GMX_trn_file":
            raise ValueError("not a TRR frame")
        off += 24
        (ir, e, box_s, vir, pres, top, sym, x_s, v_s, f_s, n, step, nre) = struct.unpack_from(">13i", data, off)
        off += 52
        t, _lam = struct.unpack_from(">ff", data, off)
        off += 8
        fr = {"step": step, "time_ps": t}
        off += ir + e
        if box_s:
            fr["box"] = np.frombuffer(data, ">f4", 9, off).reshape(3, 3)
            off += box_s
        off += vir + pres + top + sym
        for key, size in (("x", x_s), ("v", v_s), ("f", f_s)):
            if size:
                fr[key] = np.frombuffer(data, ">f4", 3 * n, off).reshape(n, 3)
                off += size
        frames.append(fr)
    return frames
