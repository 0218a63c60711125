"""Build and run the C++17/OpenMP restatement of the reference CPU MD step.

TEST INFRASTRUCTURE ONLY: the timed CPU baseline and the reference arm of
bench.py.  The binary is compiled for the machine it runs on (-march=native)
into oracle/cpu_ref/_build/, keyed by host, and never shipped.
"""
import hashlib
import json
import os
import platform
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpu_ref.cpp")
BUILD = os.path.join(HERE, "_build")


def _host_key():
    try:
        flags = open("/proc/cpuinfo").read().split("flags")[1].split("\n")[0]
    except Exception:
        flags = ""
    h = hashlib.sha1((platform.node() + platform.machine() + flags).encode()).hexdigest()[:12]
    return h


def binary_path():
    return os.path.join(BUILD, f"cpu_ref_{_host_key()}.bin")


def build(force=False):
    out = binary_path()
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(SRC):
        return out
    os.makedirs(BUILD, exist_ok=True)
    subprocess.run(["g++", "-O3", "-march=native", "-fopenmp", "-std=c++17", "-o", out + ".tmp", SRC],
                   check=True)
    os.replace(out + ".tmp", out)
    return out


def write_input(path, sysd, workload, steps, warmup, dt=0.002, skin=4.0, seed=0):
    wp = np.ascontiguousarray(np.asarray(sysd["water_pos"], np.float32).reshape(-1))
    wv = np.ascontiguousarray(np.asarray(sysd["water_vel"], np.float32).reshape(-1))
    n = len(wp) // 9
    integ = 0 if workload["integrator"] == "langevin" else 1
    from scipy.special import erfcinv
    alpha = float(erfcinv(1e-5) / workload["cutoff"])
    with open(path, "wb") as f:
        np.array([n, integ, steps, warmup], np.int32).tofile(f)
        np.concatenate([np.asarray(sysd["box_lo"], np.float32), np.asarray(sysd["box_hi"], np.float32)]).tofile(f)
        np.array([workload["cutoff"], workload["cutoff"], alpha, skin], np.float32).tofile(f)
        np.array(workload["grid"], np.int32).tofile(f)
        np.array([dt], np.float32).tofile(f)
        np.array([1.0, 300.0, 0.1], np.float32).tofile(f)
        wp.tofile(f)
        wv.tofile(f)
        ap = np.asarray(sysd.get("atom_pos", np.zeros((0, 3))), np.float32).reshape(-1, 3)
        na = len(ap)
        np.array([na], np.int32).tofile(f)
        if na:
            ap.tofile(f)
            np.asarray(sysd["atom_vel"], np.float32).reshape(-1).tofile(f)
            for k in ("atom_mass", "atom_q", "atom_sigma", "atom_eps"):
                np.asarray(sysd[k], np.float32).tofile(f)
            for k, width in (("excl", 2), ("pair14", 2)):
                a = np.asarray(sysd.get(k, np.zeros((0, width))), np.uint32).reshape(-1, width)
                np.array([len(a)], np.int32).tofile(f)
                a.tofile(f)
            for k, width, par in (("bonds", 2, ("bond_k", "bond_r0")), ("angles", 3, ("angle_k", "angle_theta0")),
                                  ("dihedrals", 4, ("dihedral_k", "dihedral_n", "dihedral_phase")),
                                  ("constraints", 2, ("constraint_r0",))):
                a = np.asarray(sysd.get(k, np.zeros((0, width))), np.uint32).reshape(-1, width)
                np.array([len(a)], np.int32).tofile(f)
                a.tofile(f)
                if len(a):
                    np.stack([np.asarray(sysd[q], np.float32) for q in par], axis=1).tofile(f)


def forces_once(sysd, cutoff, grid):
    """One force evaluation of the restatement (its first step's forces:
    O(N^2) list, flat-pair forces, bonded terms, SPME with the 1-4 vacuum
    correction), for checking it against the float64 oracle.  Returns
    f_water (nw, 4, 3) [O, H0, H1, M], f_atoms (na, 3), e_recip (self
    term included) and the pair virial."""
    binp = build()
    wl = {"integrator": "verlet", "cutoff": float(cutoff), "grid": list(grid)}
    with tempfile.TemporaryDirectory() as td:
        inp, out = os.path.join(td, "in.bin"), os.path.join(td, "f.bin")
        write_input(inp, sysd, wl, 1, 0)
        r = subprocess.run([binp, inp, "0", out], capture_output=True, text=True,
                           env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1)), timeout=600)
        if r.returncode != 0:
            raise RuntimeError(f"cpu_ref failed: {r.stderr[-500:]}")
        raw = open(out, "rb").read()
    nw, na = np.frombuffer(raw[:8], np.int32)
    d = np.frombuffer(raw[8:], np.float64)
    fw = d[:12 * nw].reshape(nw, 4, 3)
    fa = d[12 * nw:12 * nw + 3 * na].reshape(na, 3)
    e_recip, vir = d[12 * nw + 3 * na:]
    return {"f_water": fw, "f_atoms": fa, "e_recip": float(e_recip), "virial_pairs": float(vir)}


def run_sample(workload, name, seconds=20.0, steps=None, warmup=None, seed=1000, sysd=None):
    """Time the restated reference CPU step on this host for about
    ``seconds`` (bounded sample of the workload) with all host threads.
    ``sysd``: the system (built from the workload when None).  Returns a
    cpu_baseline dict."""
    from dynamics_b200 import synth
    binp = build()
    if sysd is None:
        if workload.get("n_res"):
            from dynamics_b200 import peptide
            sysd, _ = peptide.solvated_system(workload["box"], workload["n_water"], n_res=workload["n_res"],
                                              seed=seed, nacl_molar=workload.get("nacl", 0.0))
        else:
            sysd = synth.water_box(workload["n_water"], workload["box"], seed=seed)
    steps = int(steps or 100000)
    warmup = int(warmup if warmup is not None else 2)
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as td:
        inp = os.path.join(td, "in.bin")
        write_input(inp, sysd, workload, steps, warmup)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="false")
        r = subprocess.run([binp, inp, str(seconds)], capture_output=True, text=True, env=env,
                           timeout=max(600.0, 20 * seconds))
    if r.returncode != 0:
        raise RuntimeError(f"cpu_ref failed: {r.stderr[-500:]}")
    res = json.loads(r.stdout.strip().splitlines()[-1])
    cpu = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                cpu = line.split(":", 1)[1].strip()
                break
    except Exception:
        pass
    return {"value": res["value"], "unit": "ns/day", "cores": res["threads"], "kind": "port",
            "sample": f"{res['steps']} steps of workload {name} after {res['warmup']} warm-up steps "
                      f"({res['seconds']:.1f} s timed; the initial O(N^2) list build untimed)",
            "steps": res["steps"], "warmup": res["warmup"], "cpu_model": cpu,
            "note": "C++17/OpenMP restatement of the reference CPU path (reference not buildable here)",
            "pairs_in_list": res["pairs"]}
