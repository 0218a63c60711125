"""dyn_nb_forces_static (device arrays, static scratch, no allocation)
against dyn_nb_forces on the same pair list and positions.

Two calls in a row with different positions check that each call starts
from cleared scratch; a repeated call checks run-to-run identity.  Collected
last so it also runs after everything else in one process.
"""
import ctypes as C

import numpy as np
import pytest

from dynamics_b200 import _lib
from dynamics_b200 import gpu_interface as gi
from dynamics_b200 import synth
from oracle import pairs as opairs

from .systems import mixed, rel_rms

pytestmark = pytest.mark.gpu

CUTOFF = 10.0
SKIN = 4.0
ALPHA = synth.ewald_alpha(CUTOFF)
FORCE_RTOL = 1e-5   # per-site force relative RMS, as in the handle-based tests
SCALAR_RTOL = 1e-5  # virial / energy


def _dev(torch, a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a)).to(dtype).cuda()


def _prepare(torch, n_dyn, n_water, pairs, pos_dyn, pw):
    """Device copies of the inputs and the output arrays of one call."""
    pos = [_dev(torch, pos_dyn.reshape(-1), torch.float32)]
    pos += [_dev(torch, pw[k].reshape(-1), torch.float32) for k in (1, 2, 3, 4)]
    n = len(pairs["tgt"])
    arrs = [_dev(torch, pairs["tgt"].astype(np.int32), torch.int32),
            _dev(torch, pairs["src"].astype(np.int32), torch.int32),
            _dev(torch, pairs["sigma"], torch.float32), _dev(torch, pairs["eps"], torch.float32),
            _dev(torch, pairs["qq"], torch.float32), _dev(torch, np.ones(n, np.float32), torch.float32),
            _dev(torch, pairs["body_tgt"], torch.uint8), _dev(torch, pairs["body_src"], torch.uint8),
            _dev(torch, pairs["flags"], torch.uint8)]
    outs = [torch.full((3 * max(m, 1),), np.nan, dtype=torch.float64, device="cuda")
            for m in (n_dyn, n_water, n_water, n_water, n_water)]
    scal = torch.full((3,), np.nan, dtype=torch.float64, device="cuda")
    return {"n_dyn": n_dyn, "n_water": n_water, "n": n, "pos": pos, "arrs": arrs, "outs": outs, "scal": scal}


def _launch(torch, prep, ext, lj_cutoff):
    """One dyn_nb_forces_static call on prepared arrays (allocates nothing
    on the Python side either)."""
    lib = _lib.lib()
    dp = lambda t: C.c_void_p(t.data_ptr())
    ext3 = (C.c_float * 3)(*[float(x) for x in ext])
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.dyn_nb_forces_static(stream, prep["n_dyn"], prep["n_water"], *[dp(p) for p in prep["pos"]],
                                  prep["n"], *[dp(a) for a in prep["arrs"]], ext3, CUTOFF, ALPHA, lj_cutoff, 0,
                                  *[dp(o) for o in prep["outs"]], dp(prep["scal"]))
    assert rc == 0, lib.dyn_last_error().decode()


def _read(torch, prep):
    torch.cuda.synchronize()
    n_dyn, n_water = prep["n_dyn"], prep["n_water"]
    f = [o.cpu().numpy() for o in prep["outs"]]
    got = np.concatenate([f[0][:3 * n_dyn]] + [f[k][:3 * n_water] for k in (1, 2, 3, 4)])
    return got, prep["scal"].cpu().numpy()


def _static_forces(torch, n_dyn, n_water, pairs, pos_dyn, pw, ext, lj_cutoff):
    lib = _lib.lib()
    dp = lambda t: C.c_void_p(t.data_ptr())
    pos = [_dev(torch, pos_dyn.reshape(-1), torch.float32)]
    pos += [_dev(torch, pw[k].reshape(-1), torch.float32) for k in (1, 2, 3, 4)]
    n = len(pairs["tgt"])
    # q_src = 1 reproduces the stored product q_tgt * q_src exactly
    arrs = [_dev(torch, pairs["tgt"].astype(np.int32), torch.int32),
            _dev(torch, pairs["src"].astype(np.int32), torch.int32),
            _dev(torch, pairs["sigma"], torch.float32), _dev(torch, pairs["eps"], torch.float32),
            _dev(torch, pairs["qq"], torch.float32), _dev(torch, np.ones(n, np.float32), torch.float32),
            _dev(torch, pairs["body_tgt"], torch.uint8), _dev(torch, pairs["body_src"], torch.uint8),
            _dev(torch, pairs["flags"], torch.uint8)]
    outs = [torch.full((3 * max(m, 1),), np.nan, dtype=torch.float64, device="cuda")
            for m in (n_dyn, n_water, n_water, n_water, n_water)]
    scal = torch.full((3,), np.nan, dtype=torch.float64, device="cuda")
    ext3 = (C.c_float * 3)(*[float(x) for x in ext])
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.dyn_nb_forces_static(stream, n_dyn, n_water, *[dp(p) for p in pos], n,
                                  *[dp(a) for a in arrs], ext3, CUTOFF, ALPHA, lj_cutoff, 0,
                                  *[dp(o) for o in outs], dp(scal))
    assert rc == 0, lib.dyn_last_error().decode()
    torch.cuda.synchronize()
    f = [o.cpu().numpy() for o in outs]
    s = scal.cpu().numpy()
    got = np.concatenate([f[0][:3 * n_dyn]] + [f[k][:3 * n_water] for k in (1, 2, 3, 4)])
    return got, s


@pytest.mark.parametrize("lj_cutoff", [0.0, CUTOFF])
def test_static_matches_handle_path_two_calls(gpu_lib, lj_cutoff):
    torch = pytest.importorskip("torch")
    sysd = mixed()
    na, nw = len(sysd["atom_pos"]), len(sysd["water_pos"])
    fp = gi.ForcesPositsGpu(na, nw, CUTOFF, ALPHA, lj_cutoff)
    pn = gi.PerNeighborGpu.build(
        fp, sysd["atom_pos"], sysd["water_pos"][:, 0], sysd["atom_q"], sysd["atom_sigma"],
        sysd["atom_eps"], sysd["box_lo"], sysd["box_hi"], SKIN, excl=sysd.get("excl"),
        pair14=sysd.get("pair14"))
    pairs = pn.get_pairs()
    ext = (sysd["box_hi"] - sysd["box_lo"]).astype(np.float32)
    pos_dyn, pw = opairs.site_positions(sysd)
    rng = np.random.default_rng(5)
    shifted_dyn = (pos_dyn + rng.normal(0, 0.05, pos_dyn.shape)).astype(np.float32)
    shifted_w = {k: (v + rng.normal(0, 0.05, v.shape)).astype(np.float32) for k, v in pw.items()}
    results = []
    for pd, pwk in ((pos_dyn, pw), (shifted_dyn, shifted_w)):
        fd, fw, vir, en = gi.force_nonbonded_gpu(fp, pn, pd, pwk, ext)
        exp = np.concatenate([fd.reshape(-1)] + [fw[k].reshape(-1) for k in (1, 2, 3, 4)])
        got, s = _static_forces(torch, na, nw, pairs, pd, pwk, ext, lj_cutoff)
        assert np.all(np.isfinite(got))
        assert rel_rms(got, exp) < FORCE_RTOL
        assert abs(s[0] - vir) <= SCALAR_RTOL * max(abs(vir), 1.0)
        assert abs(s[1] - en) <= SCALAR_RTOL * max(abs(en), 1.0)
        assert s[2] == 0.0
        results.append(got)
    # the two position sets give different forces, so a stale accumulator shows
    assert rel_rms(results[0], results[1]) > 1e-3
    again, _ = _static_forces(torch, na, nw, pairs, shifted_dyn, shifted_w, ext, lj_cutoff)
    np.testing.assert_array_equal(again, results[1])
    fp.close()


def _handle_pairs(sysd, lj_cutoff=0.0):
    na, nw = len(sysd["atom_pos"]), len(sysd["water_pos"])
    fp = gi.ForcesPositsGpu(na, nw, CUTOFF, ALPHA, lj_cutoff)
    pn = gi.PerNeighborGpu.build(
        fp, sysd["atom_pos"], sysd["water_pos"][:, 0], sysd["atom_q"], sysd["atom_sigma"],
        sysd["atom_eps"], sysd["box_lo"], sysd["box_hi"], SKIN, excl=sysd.get("excl"),
        pair14=sysd.get("pair14"))
    pairs = pn.get_pairs()
    fp.close()
    return pairs


def test_static_allocates_nothing_and_skips_bad_pairs(gpu_lib):
    """After a first call (the device's set-up), a call leaves the device's
    free memory unchanged.  A pair with a body code above 4 and one whose
    index lies beyond its body's sites are counted in scalars[2] and
    skipped: the forces equal those of the list without them."""
    torch = pytest.importorskip("torch")
    sysd = mixed()
    na, nw = len(sysd["atom_pos"]), len(sysd["water_pos"])
    pairs = _handle_pairs(sysd)
    bad = {k: np.concatenate([v, v[:2]]) for k, v in pairs.items()}
    bad["body_tgt"][-2] = 7                  # no such body
    bad["body_tgt"][-1] = 0                  # a non-water atom ...
    bad["tgt"][-1] = na + 5                  # ... beyond the last one
    ext = (sysd["box_hi"] - sysd["box_lo"]).astype(np.float32)
    pos_dyn, pw = opairs.site_positions(sysd)
    good_p = _prepare(torch, na, nw, pairs, pos_dyn, pw)
    bad_p = _prepare(torch, na, nw, bad, pos_dyn, pw)
    _launch(torch, good_p, ext, 0.0)  # set-up of the device happens here at the latest
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    _launch(torch, bad_p, ext, 0.0)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    got_good, s_good = _read(torch, good_p)
    got_bad, s_bad = _read(torch, bad_p)
    assert s_good[2] == 0.0 and s_bad[2] == 2.0, (s_good, s_bad)
    np.testing.assert_array_equal(got_bad, got_good)
    assert abs(s_bad[0] - s_good[0]) <= SCALAR_RTOL * max(abs(s_good[0]), 1.0)


def test_static_rejects_oversize(gpu_lib):
    lib = _lib.lib()
    ext3 = (C.c_float * 3)(30.0, 30.0, 30.0)
    nw = _lib.DYN_NB_STATIC_MAX_SITES // 4 + 1
    null = C.c_void_p(0)
    rc = lib.dyn_nb_forces_static(null, 0, nw, *([null] * 5), 0, *([null] * 9), ext3, CUTOFF, ALPHA,
                                  0.0, 0, *([null] * 5), C.c_void_p(1))
    assert rc == _lib.DYN_ERR_INVALID
    assert b"DYN_NB_STATIC_MAX_SITES" in lib.dyn_last_error()
