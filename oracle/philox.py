"""Philox4x32-10 counter-based RNG (oracle twin of the CUDA engine's RNG).

Published method: Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
easy as 1, 2, 3", SC'11.  The reference draws from an unseeded ThreadRng
(src/barostat.rs:319, src/thermostat.rs:276-279,324-360), so its noise
streams are irreproducible; the engine replaces them with this seeded stream
and the oracle reproduces it bit for bit, which makes stochastic steps
comparable between the GPU and the oracle.

Counter layout used by the engine (every field uint32):
  Langevin OU noise for a particle : (particle_id, step_lo, STREAM_OU, step_hi)
  CSVR draws (attempt a)           : (a,           step_lo, STREAM_CSVR, step_hi)
  C-rescale draw                   : (0,           step_lo, STREAM_BARO, step_hi)
Key = (seed_lo, seed_hi).
"""
import numpy as np

M0 = np.uint64(0xD2511F53)
M1 = np.uint64(0xCD9E8D57)
W0 = np.uint32(0x9E3779B9)
W1 = np.uint32(0xBB67AE85)
MASK = np.uint64(0xFFFFFFFF)

STREAM_OU = 1
STREAM_CSVR = 2
STREAM_BARO = 3
STREAM_INIT = 4


def philox4x32(c0, c1, c2, c3, k0, k1, rounds=10):
    """Vectorised Philox4x32; all inputs broadcastable uint32 arrays."""
    c0 = np.asarray(c0, dtype=np.uint32).astype(np.uint64)
    c1 = np.asarray(c1, dtype=np.uint32).astype(np.uint64)
    c2 = np.asarray(c2, dtype=np.uint32).astype(np.uint64)
    c3 = np.asarray(c3, dtype=np.uint32).astype(np.uint64)
    k0 = np.asarray(k0, dtype=np.uint32).astype(np.uint64)
    k1 = np.asarray(k1, dtype=np.uint32).astype(np.uint64)
    c0, c1, c2, c3, k0, k1 = np.broadcast_arrays(c0, c1, c2, c3, k0, k1)
    c0, c1, c2, c3, k0, k1 = (a.copy() for a in (c0, c1, c2, c3, k0, k1))
    for r in range(rounds):
        p0 = M0 * c0
        p1 = M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & MASK, lo1, (hi0 ^ c3 ^ k1) & MASK, lo0
        if r != rounds - 1:
            k0 = (k0 + np.uint64(W0)) & MASK
            k1 = (k1 + np.uint64(W1)) & MASK
    return (c0.astype(np.uint32), c1.astype(np.uint32), c2.astype(np.uint32),
            c3.astype(np.uint32))


def uniform24(x):
    """(x >> 8) + 0.5 scaled to (0, 1); exact in float32 and float64."""
    return ((np.asarray(x, dtype=np.uint32) >> np.uint32(8)).astype(np.float64) + 0.5) * (2.0 ** -24)


def normals4(c0, c1, c2, c3, seed):
    """Four standard normals per counter via Box-Muller on 24-bit uniforms."""
    k0 = np.uint32(seed & 0xFFFFFFFF)
    k1 = np.uint32((seed >> 32) & 0xFFFFFFFF)
    x0, x1, x2, x3 = philox4x32(c0, c1, c2, c3, k0, k1)
    out = []
    for a, b in ((x0, x1), (x2, x3)):
        u = uniform24(a)
        v = uniform24(b)
        r = np.sqrt(-2.0 * np.log(u))
        out.append(r * np.cos(2.0 * np.pi * v))
        out.append(r * np.sin(2.0 * np.pi * v))
    return out


def step_words(step):
    step = int(step)
    return np.uint32(step & 0xFFFFFFFF), np.uint32((step >> 32) & 0xFFFFFFFF)


def ou_normals(particle_ids, step, seed):
    """(n, 3) standard normals for the Langevin OU kick of ``particle_ids``."""
    lo, hi = step_words(step)
    n0, n1, n2, _ = normals4(np.asarray(particle_ids, dtype=np.uint32), lo, STREAM_OU, hi, seed)
    return np.stack([n0, n1, n2], axis=-1)


def gamma_marsaglia_tsang(shape, step, seed, stream=STREAM_CSVR, max_attempts=64):
    """Gamma(shape, 1) by Marsaglia & Tsang (ACM TOMS 26, 2000), shape >= 1.

    Attempt a draws from counter (a + 1, step_lo, stream, step_hi): normal x
    from the first Box-Muller output, uniform from word 2.  Returns the
    accepted value, or d (the mode) if no attempt was accepted.
    """
    lo, hi = step_words(step)
    d = shape - 1.0 / 3.0
    c = 1.0 / np.sqrt(9.0 * d)
    k0 = np.uint32(seed & 0xFFFFFFFF)
    k1 = np.uint32((seed >> 32) & 0xFFFFFFFF)
    for a in range(max_attempts):
        x0, x1, x2, x3 = philox4x32(np.uint32(a + 1), lo, np.uint32(stream), hi, k0, k1)
        u1 = float(uniform24(x0))
        u2 = float(uniform24(x1))
        x = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
        v = (1.0 + c * x) ** 3
        if v <= 0.0:
            continue
        u = float(uniform24(x2))
        if np.log(u) < 0.5 * x * x + d - d * v + d * np.log(v):
            return d * v
    return d


def csvr_normal(step, seed, stream=STREAM_CSVR):
    """The N(0,1) draw of the CSVR update: counter (0, step_lo, stream, step_hi)."""
    lo, hi = step_words(step)
    n0, _, _, _ = normals4(np.uint32(0), lo, np.uint32(stream), hi, seed)
    return float(n0)
