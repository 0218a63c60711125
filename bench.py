"""Benchmark: ns/day of the device-resident MD step on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
                    [--impl ours|reference]

A "step" is one full MD step (MdState::step, src/integrate.rs:72) of the
workload: integration, neighbour-list upkeep, short-range pairs, SPME on the
reference's every-2-steps schedule, thermostat/barostat.  Inputs are
seeded synthetic systems (no dataset) of the configured shapes.  K timed
steps are each bracketed by CUDA events on the engine's stream, with a
256 MiB L2 flush between steps (outside the brackets), so every step starts
with a cold L2.  Under torchrun each rank runs an independent replica
(weak scaling, no collective on the data path) and rank 0 prints the line.

--impl reference times the C++17/OpenMP restatement of the reference's CPU
path (oracle/cpu_ref) on the host cores for a bounded sample of the same
workload.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))


def clock_csv(rank):
    """Where the nvidia-smi clock samples of the timed region go: the
    directory named by DYNB200_OUT, else /tmp."""
    out = os.environ.get("DYNB200_OUT") or "/tmp"
    return os.path.join(out, f"clocks_rank{rank}.csv")
sys.path.insert(0, ROOT)

WORKLOADS = {
    # 512 OPC waters, 24.8 A cube, rc 10, 32^3, Langevin-middle gamma 1/ps
    "c1": dict(n_water=512, box=24.8, cutoff=10.0, grid=(32, 32, 32), integrator="langevin",
               barostat=False),
    # ~100k atoms: 24,000 OPC waters in a 98 A cube, rc 10, 96^3, CSVR 300 K + C-rescale 1 bar
    # ~32k atoms: a 40-residue ff19SB peptide, counter-ions, 7,800 OPC waters
    # in a 62 A cube, rc 9, 64^3, CSVR 300 K, bond-to-H constraints
    "c2": dict(n_water=7800, box=62.0, cutoff=9.0, grid=(64, 64, 64), integrator="vv_csvr",
               barostat=False, n_res=(40,), nacl=0.0),
    # ~100k atoms: a 300-residue ff19SB peptide, 24,000 OPC waters with NaCl
    # at 0.15 M (plus counter-ions; ions replace waters) in a 98 A cube,
    # rc 10, 96^3, CSVR 300 K + C-rescale 1 bar, bond-to-H constraints
    "c3": dict(n_water=24000, box=98.0, cutoff=10.0, grid=(96, 96, 96), integrator="vv_csvr",
               barostat=True, n_res=(300,), nacl=0.15),
    # the same box with water only
    "c3w": dict(n_water=24000, box=98.0, cutoff=10.0, grid=(96, 96, 96), integrator="vv_csvr",
                barostat=True),
    # batched form: 64 water boxes, 512-8000 waters log-uniform, 0.0334 / A^3,
    # rc 9, grid ~1 A (FFT-friendly), Langevin-middle 300 K; one launch per
    # stage for all 64 (compared with the same systems one by one)
    "c4w": dict(kind="batch", n_sys=64, cutoff=9.0, integrator="langevin", barostat=False,
                n_water=None),
    # serving form: Poisson arrivals (20 / s) of systems drawn from the c4w
    # size distribution, 5000 steps each, Langevin-middle 300 K, 150 GB budget
    "c5w": dict(kind="serve", n_req=400, rate=20.0, steps_each=5000, cutoff=9.0, budget=150e9,
                integrator="langevin", barostat=False, n_water=None),
    # as c4w / c5w with 0-3 ten-residue ff19SB peptides (and counter-ions,
    # bond-to-H constraints) in every member
    "c4": dict(kind="batch", n_sys=64, cutoff=9.0, integrator="langevin", barostat=False,
               n_water=None, peptides=3),
    "c5": dict(kind="serve", n_req=400, rate=20.0, steps_each=5000, cutoff=9.0, budget=150e9,
               integrator="langevin", barostat=False, n_water=None, peptides=3),
}
DEFAULT_WORKLOAD = "c3"
DT = 0.002


def build_system(name, seed):
    from dynamics_b200 import md, synth
    w = WORKLOADS[name]
    if w.get("n_res"):
        from dynamics_b200 import peptide
        sysd, _ = peptide.solvated_system(w["box"], w["n_water"], n_res=w["n_res"], seed=seed,
                                          nacl_molar=w.get("nacl", 0.0))
    else:
        sysd = synth.water_box(w["n_water"], w["box"], seed=seed)
    alpha = synth.ewald_alpha(w["cutoff"])
    cfg = md.MdConfig(coulomb_cutoff=w["cutoff"], lj_cutoff=w["cutoff"], spme_alpha=alpha,
                      spme_grid=w["grid"], seed=seed)
    if w["integrator"] == "langevin":
        cfg.integrator = md.LangevinMiddle(gamma=1.0)
    else:
        cfg.integrator = md.VerletVelocity(thermostat=0.1)
    if w["barostat"]:
        cfg.barostat_cfg = md.BarostatCfg(pressure_target=1.0, tau=5.0, solvent_compressibility=4.5e-5)
    return sysd, _override(cfg)


def _member_job(job):
    """One batched / served member (run in a worker process): a water box,
    or a box with n_pep ten-residue peptides."""
    n_water, n_pep, seed = job
    from dynamics_b200 import synth
    if n_pep is not None:
        from dynamics_b200 import peptide
        sysd, grid, _ = peptide.batch_member(int(n_water), int(n_pep), seed=seed)
        return sysd, grid
    return synth.batch_member(int(n_water), seed=seed)


def build_members(w, sizes, seeds, rng):
    """Members for the given sizes and seeds; with w["peptides"], each gets
    0..w["peptides"] peptides (counts drawn from rng here, so the result does
    not depend on the workers).  Built in parallel on the host cores by
    spawned processes (no CUDA state is inherited)."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    jobs = [(int(n), int(rng.integers(0, w["peptides"] + 1)) if w.get("peptides") else None, int(sd))
            for n, sd in zip(sizes, seeds)]
    workers = max(1, min(len(jobs), (os.cpu_count() or 1)))
    if workers == 1 or len(jobs) < 4:
        return [_member_job(j) for j in jobs]
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_member_job, jobs, chunksize=max(1, len(jobs) // (4 * workers))))


# MdConfig fields set from the command line (--set field=value), applied to
# every system a workload builds
CFG_OVERRIDES = {}


def _override(cfg):
    for k, val in CFG_OVERRIDES.items():
        if not hasattr(cfg, k):
            raise SystemExit(f"--set: MdConfig has no field {k!r}")
        setattr(cfg, k, type(getattr(cfg, k))(val))
    return cfg


def build_batch(name, seed):
    from dynamics_b200 import md, synth
    w = WORKLOADS[name]
    sizes = synth.config4_sizes(w["n_sys"], seed=seed)
    rng = np.random.default_rng(seed + 7919)
    systems, cfgs = [], []
    alpha = synth.ewald_alpha(w["cutoff"])
    built = build_members(w, sizes, [seed * 1000 + i for i in range(len(sizes))], rng)
    for i, (sysd, grid) in enumerate(built):
        cfg = md.MdConfig(coulomb_cutoff=w["cutoff"], lj_cutoff=w["cutoff"], spme_alpha=alpha,
                          spme_grid=grid, seed=seed * 1000 + i,
                          integrator=md.LangevinMiddle(gamma=1.0))
        systems.append(sysd)
        cfgs.append(_override(cfg))
    return systems, cfgs


def measure_batch(name, args, stream, dev, dist=None, rank=0, world=1):
    """Batched form: aggregate ns/day of all members advanced together
    (CUDA events around each batched step, 256 MiB L2 flush between steps),
    against the same systems stepped one by one through the plain path, and
    the end-to-end rate with every member's state in and out through host
    memory each step.  Returns the fields of a JSON line."""
    import torch

    from dynamics_b200 import md
    w = WORKLOADS[name]
    systems, cfgs = build_batch(name, seed=1 + rank)
    systems = [md.equilibrate(s, c, n_steps=min(args.equil, 200), dt=0.001) for s, c in zip(systems, cfgs)]
    n_sys = len(systems)
    n_water = int(sum(len(s["water_pos"]) for s in systems))
    n_atoms = int(sum(len(s.get("atom_pos", ())) for s in systems))
    steps = max(args.steps, 50)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    # ---- plain path, one system at a time (each its own graph per step) ----
    k_plain = max(10, min(steps, 100))
    plain_ms = 0.0
    for sysd, c in zip(systems, cfgs):
        st = md.MdState(sysd, c, stream=stream.cuda_stream)
        st.step(DT, args.warmup)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        st.step(DT, k_plain)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        plain_ms += e0.elapsed_time(e1) / k_plain
        st.close()
    # ---- batched ----
    batch = md.MdBatch(systems, cfgs, stream=stream.cuda_stream)
    batch.step(DT, args.warmup)
    torch.cuda.synchronize(dev)
    r0 = sum(m.energies()["list_rebuilds"] for m in batch.members)
    p0 = sum(m.energies()["list_prunes"] for m in batch.members)
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    clocks = ClockSampler(clock_csv(rank) + ".batch")
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with clocks:
        for k in range(steps):
            flush.zero_()
            ev0[k].record(stream)
            batch.step(DT, 1)
            ev1[k].record(stream)
        torch.cuda.synchronize(dev)
    batch.sync()
    ms = max_over_ranks(float(np.sum([ev0[k].elapsed_time(ev1[k]) for k in range(steps)])), dist, dev)
    rebuilds = sum(m.energies()["list_rebuilds"] for m in batch.members) - r0
    prunes = sum(m.energies()["list_prunes"] for m in batch.members) - p0
    fixed_s, reb_k, per_k = batch.launches(True)
    fixed_n, _, _ = batch.launches(False)
    # the batch's rebuild (and prune, 2 kernels) IF nodes fire on a step
    # where any member needs them: at most one of each per step
    launches = ((fixed_s + fixed_n) / 2.0 * steps + reb_k * min(rebuilds, steps)
                + 2 * min(max(0, prunes - rebuilds), steps))
    value = aggregate_ns_per_day(steps, n_sys, world, ms)
    plain_value = DT * 1e-3 * n_sys / (plain_ms * 1e-3) * 86400.0
    # ---- the same members with the autotuner's choices (--tune) ----
    tuned = None
    if getattr(args, "tune", False):
        from dynamics_b200 import tune as _tune
        t0 = time.perf_counter()
        tb = md.MdBatch(systems, cfgs, stream=stream.cuda_stream, tune=True)
        tune_s = time.perf_counter() - t0
        tb.step(DT, args.warmup)
        torch.cuda.synchronize(dev)
        for k in range(steps):
            flush.zero_()
            ev0[k].record(stream)
            tb.step(DT, 1)
            ev1[k].record(stream)
        torch.cuda.synchronize(dev)
        tb.sync()
        tms = max_over_ranks(float(np.sum([ev0[k].elapsed_time(ev1[k]) for k in range(steps)])), dist, dev)
        keys = sorted({_tune.size_class(sd, c) for sd, c in zip(systems, cfgs)})
        tuned = {"value": round(aggregate_ns_per_day(steps, n_sys, world, tms), 2),
                 "ms_per_step": round(tms / steps, 5), "over_untuned": round(ms / tms, 3),
                 "tune_s": round(tune_s, 1), "classes": {k: _tune.lookup(k) for k in keys}}
        tb.close()
    # ---- end to end: every member's positions/velocities in and out per step,
    # one copy each way for the whole batch through its page-locked area ----
    host = batch.host_buffer()
    batch.step_host(DT, 1, None, host)
    n_e2e = max(5, steps // 10)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        batch.step_host(DT, 1, host, host)
    t_e2e = time.perf_counter() - t0
    e2e_value = n_e2e * DT * 1e-3 * n_sys * world / t_e2e * 86400.0
    io_bytes = int(host.nbytes)
    batch.close()
    return {
        "value": round(value, 2), "unit": "ns/day (aggregate over members)", "steps": steps,
        "warmup": args.warmup, "ms_per_step": round(ms / steps, 5),
        "members": n_sys, "n_water_total": n_water, "n_atoms_total": n_atoms,
        "member_steps_per_s": round(n_sys * steps / (ms * 1e-3), 1),
        "plain_one_by_one": {"value": round(plain_value, 2), "unit": "ns/day (aggregate)",
                             "ms_per_round": round(plain_ms, 4), "steps_each": k_plain},
        "batch_over_plain": round(value / world / plain_value, 3),
        "tuned": tuned,
        "e2e": {"value": round(e2e_value, 2), "unit": "ns/day (aggregate)",
                "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes,
                "of_device": round(e2e_value / value, 3), "path": "dyn_batch_step_host"},
        "gpu_launches": int(round(launches)),
        "launches_per_step": {"spme": fixed_s, "no_spme": fixed_n, "rebuild_extra": reb_k, "periodic_extra": per_k},
        "clocks": clocks.summary(0 if dev.index is None else dev.index),
        "data": "synthetic (seeded OPC water boxes" + (", 0-3 ten-residue ff19SB peptides each"
                                                        if w.get("peptides") else "")
                + ", equilibrated on device)",
        "config": {"workload": name, "sizes": "512-8000 waters, log-uniform", "cutoff_A": w["cutoff"],
                   "grid": "FFT-friendly ~1 A", "integrator": "langevin_middle", "dt_fs": DT * 1e3,
                   "l2": "256 MiB flush between timed steps"},
    }


def serve_requests(name, n_req, rate, steps_each, seed, pool_size, args):
    """A Poisson(rate) stream of n_req requests, each a system drawn from a
    pool of pool_size systems whose sizes follow the workload's size
    distribution (built and equilibrated once), steps_each steps each."""
    from dynamics_b200 import md, serve, synth
    w = WORKLOADS[name]
    sizes = synth.config4_sizes(pool_size, seed=seed)
    rng = np.random.default_rng(seed + 7919)
    built = build_members(w, sizes, [seed * 1000 + i for i in range(pool_size)], rng)
    alpha = synth.ewald_alpha(w["cutoff"])
    pool = []
    for i, (sysd, grid) in enumerate(built):
        cfg = md.MdConfig(coulomb_cutoff=w["cutoff"], lj_cutoff=w["cutoff"], spme_alpha=alpha, spme_grid=grid,
                          seed=seed * 1000 + i, integrator=md.LangevinMiddle(gamma=1.0))
        pool.append((md.equilibrate(sysd, cfg, n_steps=min(args.equil, 200), dt=0.001), cfg))
    pick = np.random.default_rng(seed + 31).integers(0, pool_size, n_req)
    arrivals = serve.poisson_arrivals(n_req, rate, seed=seed)
    return pool, [(int(k), float(t)) for k, t in zip(pick, arrivals)]


def serve_once(pool, stream_spec, steps_each, budget, max_members, stream):
    from dynamics_b200 import md, serve
    reqs = []
    for rid, (k, t) in enumerate(stream_spec):
        sysd, cfg = pool[k]
        c = md.MdConfig(**{**cfg.__dict__, "seed": cfg.seed + 1000 * rid})
        reqs.append(serve.Request(rid=rid, system=sysd, cfg=c, n_steps=steps_each, arrival=t))
    srv = serve.Server(budget_bytes=budget, max_members=max_members, round_steps=100, dt=DT, stream=stream,
                       keep_states=False)
    rep = srv.run(reqs)
    return {"value": round(rep.ns_per_day, 2), "unit": "ns/day (aggregate over requests)",
            "latency_s": {k: round(v, 4) for k, v in rep.latency_s.items()},
            "queue_wait_s": {k: round(v, 4) for k, v in rep.queue_wait_s.items()},
            "wall_s": round(rep.wall_s, 3), "requests": len(reqs), "peak_members": rep.peak_members,
            "peak_device_GB": round(rep.peak_bytes / 1e9, 3), "budget_waits": rep.budget_waits,
            "member_steps": rep.steps_total}


def measure_served(name, args, stream, capacity_req_per_s=None, n_req=400, steps_each=1000, pool_size=64,
                   budget=0.7e9):
    """Serving form: continuous batching of a Poisson stream at the workload's
    rate (20 / s) and at a sustainable rate (half the measured batched
    capacity), under a device-memory budget small enough to hold requests
    back (0.7 GB: unconstrained, the 20 / s stream peaks near 1.2 GB), against
    a real server run one request at a time."""
    w = WORKLOADS[name]
    rate = w["rate"]
    pool, spec = serve_requests(name, n_req, rate, steps_each, 7, pool_size, args)
    out = {"stream": {"requests": n_req, "steps_each": steps_each, "arrival_rate_per_s": rate,
                      "pool": f"{pool_size} systems drawn from the c4 size distribution, equilibrated once; "
                              "each request one of them with its own seed",
                      "budget_GB": budget / 1e9, "round_steps": 100}}
    out["at_rate"] = serve_once(pool, spec, steps_each, budget, 256, stream)
    if capacity_req_per_s is None:
        capacity_req_per_s = out["at_rate"]["member_steps"] / out["at_rate"]["wall_s"] / steps_each
    sus = max(1.0, 0.5 * capacity_req_per_s)
    from dynamics_b200 import serve
    arr = serve.poisson_arrivals(n_req, sus, seed=8)
    spec_s = [(k, float(t)) for (k, _), t in zip(spec, arr)]
    out["sustainable"] = serve_once(pool, spec_s, steps_each, budget, 256, stream)
    out["sustainable"]["arrival_rate_per_s"] = round(sus, 3)
    out["one_at_a_time"] = serve_once(pool, spec, steps_each, budget, 1, stream)
    out["one_at_a_time"]["note"] = "the same stream at the workload's rate, served by a server holding one member"
    out["served_over_one_at_a_time"] = round(out["at_rate"]["value"] / out["one_at_a_time"]["value"], 3)
    return out


def run_batch(args):
    """--workload c4 / c4w: the batched form's own JSON line."""
    import torch
    rank, world, local, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    res = measure_batch(args.workload, args, stream, dev, dist, rank, world)
    if dist:
        dist.barrier()
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    out = {"metric": "ns/day", "value": res["value"], "unit": res["unit"], "n_gpus": world, "steps": res["steps"],
           "warmup": args.warmup, "ms_per_step": res["ms_per_step"], "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": res["data"],
           "config": {**res["config"], "members": res["members"], "parallelism": f"replicas x{world}"},
           **{k: res[k] for k in ("plain_one_by_one", "batch_over_plain", "tuned", "e2e", "gpu_launches",
                                  "launches_per_step", "clocks", "n_water_total", "n_atoms_total")},
           "cpu_baseline": None}
    print(json.dumps(out))
    if dist:
        dist.destroy_process_group()


def run_serve(args):
    """--workload c5 / c5w: the serving form's own JSON line."""
    import torch
    rank, world, local, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    w = WORKLOADS[args.workload]
    clocks = ClockSampler(clock_csv(rank))
    with clocks:
        res = measure_served(args.workload, args, stream.cuda_stream, n_req=w["n_req"], steps_each=w["steps_each"],
                             budget=w["budget"])
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    a = res["at_rate"]
    out = {"metric": "ns/day", "value": a["value"], "unit": a["unit"], "n_gpus": world,
           "steps": a["member_steps"], "warmup": args.warmup,
           "ms_per_step": round(a["wall_s"] * 1e3 / max(1, a["member_steps"]), 6),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded OPC water boxes" + (", 0-3 ten-residue ff19SB peptides each"
                                                           if w.get("peptides") else "") + ")",
           "config": {"workload": args.workload, "parallelism": f"replicas x{world}", **res["stream"]},
           "served": res, "e2e": {"value": a["value"], "unit": a["unit"], "h2d_bytes_per_step": None,
                                  "d2h_bytes_per_step": None,
                                  "note": "inputs enter through the public API at admission and results leave "
                                          "at completion, inside the served wall time"},
           "clocks": clocks.summary(local), "cpu_baseline": None}
    print(json.dumps(out))
    if dist:
        dist.destroy_process_group()


def count_pairs(sysd, cutoff):
    """Interacting site pairs within the cutoff (the algorithmic pair count):
    LJ pairs between LJ sites (water O, atoms with eps > 0) and Coulomb pairs
    between charged sites, not in the same water and not excluded (1-2, 1-3;
    1-4 pairs count once, as scaled pairs)."""
    from scipy.spatial import cKDTree
    lo = np.asarray(sysd["box_lo"], np.float64)
    ext = (np.asarray(sysd["box_hi"], np.float64) - lo)
    wp = np.asarray(sysd["water_pos"], np.float64)
    nw = len(wp)
    o = wp[:, 0]
    bis = (wp[:, 1] - o) + (wp[:, 2] - o)
    m = o + bis / np.linalg.norm(bis, axis=1, keepdims=True) * 0.15939833
    ap = np.asarray(sysd.get("atom_pos", np.zeros((0, 3))), np.float64).reshape(-1, 3)
    na = len(ap)
    excl = set()
    if na and "excl" in sysd and len(sysd["excl"]):
        excl = set(map(tuple, np.sort(np.asarray(sysd["excl"], np.int64), axis=1).tolist()))

    def npairs(pts, mol, atom_id):
        """(pairs, water-water pairs) within the cutoff."""
        t = cKDTree(np.mod(pts - lo, ext), boxsize=ext)
        p = t.query_pairs(cutoff, output_type="ndarray")
        keep = mol[p[:, 0]] != mol[p[:, 1]]
        p = p[keep]
        n_ww = int(np.count_nonzero((mol[p[:, 0]] >= 0) & (mol[p[:, 1]] >= 0)))
        if excl:
            a, b = atom_id[p[:, 0]], atom_id[p[:, 1]]
            both = (a >= 0) & (b >= 0)
            if both.any():
                pa = np.sort(np.stack([a[both], b[both]], 1), axis=1)
                ex = np.array([tuple(x) in excl for x in pa.tolist()])
                return int(len(p) - np.count_nonzero(ex)), n_ww
        return int(len(p)), n_ww

    ljm = np.asarray(sysd.get("atom_eps", np.zeros(na))) > 0
    qm = np.asarray(sysd.get("atom_q", np.zeros(na))) != 0
    amol = -1 - np.arange(na)
    aid = np.arange(na)
    lj_pts = np.concatenate([o, ap[ljm]])
    lj_mol = np.concatenate([np.arange(nw), amol[ljm]])
    lj_id = np.concatenate([np.full(nw, -1), aid[ljm]])
    n_lj, n_lj_ww = npairs(lj_pts, lj_mol, lj_id)
    q_pts = np.concatenate([wp[:, 1], wp[:, 2], m, ap[qm]])
    q_mol = np.concatenate([np.tile(np.arange(nw), 3), amol[qm]])
    q_id = np.concatenate([np.full(3 * nw, -1), aid[qm]])
    n_c, n_c_ww = npairs(q_pts, q_mol, q_id)
    return {"lj": n_lj, "coulomb": n_c, "lj_ww": n_lj_ww, "coulomb_ww": n_c_ww}


class ClockSampler:
    """SM clocks and clock-event reasons sampled DURING a timed region: an
    in-process thread reads NVML every 10 ms (read-only queries), so even a
    region of a few milliseconds gets samples; nvidia-smi -lms 200 is the
    fallback when NVML is unavailable.  Rows go to ``path`` as CSV."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, path, device_index=None):
        self.path = path
        self.proc = None
        self.thread = None
        self.rows = []
        self.device_index = device_index

    def _nvml_loop(self, nv, h, index):
        import threading
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                self.rows.append([str(index), str(sm), str(mx), f"{pw:.1f}", hex(rs)] +
                                 ["Active" if rs & getattr(nv, c) else "Not Active" for _, c in self.REASONS])
            except Exception:
                pass
            self.stop.wait(0.01)

    def __enter__(self):
        import threading
        index = self.device_index
        if index is None:
            try:
                import torch
                index = torch.cuda.current_device()
            except Exception:
                index = 0
        self.index = index
        try:
            import pynvml as nv
            nv.nvmlInit()
            # the physical GPU behind this process's device index
            vis = [x.strip() for x in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if x.strip()]
            ident = vis[index] if index < len(vis) else str(index)
            if ident.startswith("GPU-"):
                h = nv.nvmlDeviceGetHandleByUUID(ident)
            else:
                h = nv.nvmlDeviceGetHandleByIndex(int(ident) if ident.isdigit() else index)
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h, index), daemon=True)
            self.thread.start()
            while not self.rows and self.thread.is_alive():
                time.sleep(0.002)  # the first sample precedes the timed region
            return self
        except Exception:
            self.thread = None
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=2)
            with open(self.path, "w") as f:
                for r in self.rows:
                    f.write(", ".join(r) + "\n")
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self, device_index):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines()]
        except Exception:
            return None
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 9 and r[0].strip() == str(device_index)]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = []
        for name, col in (("hw_slowdown", 5), ("hw_thermal_slowdown", 6), ("sw_thermal_slowdown", 7),
                          ("sw_power_cap", 8)):
            if any(r[col].lower().startswith("active") for r in rows):
                reasons.append(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(n_gpus, backend="nccl"):
    """Rank, world size, local rank and the torch.distributed module (None
    for one process) of a run launched one process per GPU; every rank runs
    an independent replica, so the only collectives are the barriers and
    the max over ranks of the timed duration."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return rank, world, local, pg


def max_over_ranks(ms, dist, device):
    """The job's timed duration: the largest of the ranks' durations."""
    if not dist:
        return ms
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_ns_per_day(steps, systems_per_rank, world, ms):
    """Simulated ns per day of the whole job: every rank advances
    systems_per_rank systems by steps steps of DT in the job's ms."""
    return steps * DT * 1e-3 * systems_per_rank * world / (ms * 1e-3) * 86400.0


def plain_config(name, cfg, n_water, n_atoms, world):
    """The config object of a plain-workload JSON line (both arms)."""
    w = WORKLOADS[name]
    return {"workload": name, "n_water": n_water, "atoms": 4 * n_water + n_atoms,
            "peptide_residues": list(w.get("n_res", ())), "nacl_molar": w.get("nacl", 0.0),
            "box_A": w["box"], "cutoff_A": w["cutoff"], "spme_grid": list(w["grid"]),
            "spme_interval": cfg.spme_interval, "dt_fs": DT * 1e3,
            "integrator": w["integrator"], "barostat": w["barostat"],
            "l2": "256 MiB flush between timed steps",
            "parallelism": f"replicas x{world}"}


def run_ours(args):
    import torch

    from dynamics_b200 import _lib, md
    rank, world, local, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # a dedicated stream: the engine, the L2 flush and the timing events
    # must share one stream (the legacy default stream cannot host graphs)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    name = args.workload
    w = WORKLOADS[name]
    sysd, cfg = build_system(name, seed=1000 + rank)
    sysd = md.equilibrate(sysd, cfg, n_steps=args.equil, dt=0.001)
    # the autotuner's choice for this size class (the shipped B200 table or
    # the user's cache), if there is one
    from dynamics_b200 import tune
    tuned_knobs = tune.lookup(tune.size_class(sysd, cfg))
    if tuned_knobs is not None:
        cfg = tune.apply_tuned(sysd, cfg)
    st = md.MdState(sysd, cfg, stream=stream.cuda_stream)
    st.step(DT, args.warmup)
    torch.cuda.synchronize(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(clock_csv(rank))
    e_before = st.energies()
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with clocks:
        t_wall = time.perf_counter()
        for k in range(args.steps):
            flush.zero_()
            ev0[k].record(stream)
            st.step(DT, 1)
            ev1[k].record(stream)
        torch.cuda.synchronize(dev)
        t_wall = time.perf_counter() - t_wall
    if dist:
        dist.barrier()
    st.sync()
    ms_steps = [ev0[k].elapsed_time(ev1[k]) for k in range(args.steps)]
    ms = max_over_ranks(float(np.sum(ms_steps)), dist, dev)
    en = st.energies()
    value = aggregate_ns_per_day(args.steps, 1, world, ms)
    # ---- stage timing and roofline of the dominant kernel ----
    stages = st.stage_times(DT, 40)
    pc = count_pairs({**sysd, "water_pos": st.state()["water_pos"]}, w["cutoff"])
    n_lj, n_c = pc["lj"], pc["coulomb"]
    # the dominant kernel: water-water pairs only, per launch
    ww_flops = pc["lj_ww"] * (19 + 15) + pc["coulomb_ww"] * (19 + 23)
    ww_ms = stages["pairs_water_water"]
    flops = n_lj * (19 + 15) + n_c * (19 + 23)   # frozen per-pair convention
    pair_ms = stages["pairs"]
    achieved = flops / (pair_ms * 1e-3) / 1e12
    import ctypes as C
    peak = C.c_double()
    _lib.check(_lib.lib().dyn_probe_fp32_peak(stream.cuda_stream, C.byref(peak)))
    # PME: algorithmic bytes of spread + gather per SPME step
    nq = 3 * st.n_water + st.n_atoms
    K = np.prod(cfg.spme_grid)
    pme_bytes = nq * 16 + K * 4 + nq * 16 + K * 4 + nq * 12
    pme_ms = stages["spme"]
    spread_bytes, gather_bytes = nq * 16 + K * 4, nq * 16 + K * 4 + nq * 12
    # ---- end-to-end through the host-buffer C-ABI step ----
    nw, na = st.n_water, st.n_atoms
    st_nw, st_na = nw, na
    pin = lambda shape: torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()
    s0 = st.state()
    io = {"water_pos": pin((nw, 3, 3)), "water_vel": pin((nw, 3, 3))}
    if na:
        io.update({"atom_pos": pin((na, 3)), "atom_vel": pin((na, 3))})
    for k in io:
        io[k][:] = s0[k][:len(io[k])]
    n_e2e = max(20, args.steps // 5)
    st.step_host(DT, 1, io, io)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        st.step_host(DT, 1, io, io)
    t_e2e = time.perf_counter() - t0
    io_bytes = int(sum(a.nbytes for a in io.values()))
    e2e_value = n_e2e * DT * 1e-3 * world / t_e2e * 86400.0
    # kernels in the timed region: every step's fixed set, plus the rebuild
    # and periodic-task kernels on the steps whose conditional nodes fired
    n_rebuild_k, n_periodic_k = st.launches_conditional()
    rebuilds = en["list_rebuilds"] - e_before["list_rebuilds"]
    s0 = e_before["step"]
    due = sum(1 for t in range(s0 + 1, s0 + args.steps + 1)
              if (cfg.zero_com_drift and t % cfg.com_removal_interval == 0)
              or (cfg.reset_angle and t % 1000 == 0)
              or (cfg.recenter_sim_box and na and t % 30 == 0))
    # a prune of the water-water lists without a rebuild adds its 2 kernels
    prune_only = max(0, (en["list_prunes"] - e_before["list_prunes"]) - rebuilds)
    launches = ((st.launches_per_step(True) + st.launches_per_step(False)) / 2.0 * args.steps
                + rebuilds * n_rebuild_k + prune_only * 2 + due * n_periodic_k)
    clk = clocks.summary(local)
    st.close()
    if dist:
        dist.barrier()
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs")
    cpu = cpu_baseline(name, args, sysd) if (world == 1 and not args.no_cpu) else None
    out = {
        "metric": "ns/day", "value": round(value, 2), "unit": "ns/day", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded ff19SB peptide / ions / OPC water, equilibrated on device)"
                if w.get("n_res") else "synthetic (seeded OPC water lattice, equilibrated on device)",
        "config": plain_config(name, cfg, st_nw, st_na, world),
        "tuned": None if tuned_knobs is None else {"knobs": tuned_knobs, "spme_grid_used": list(cfg.spme_grid),
                                                  "source": "dynamics_b200/data/tune_b200.json or the user cache"},
        "roofline": roofline_dominant(name, ww_flops, ww_ms, peak.value, pc),
        "roofline_pair_stage": {"bound": "fp32", "kernel": "all short-range pair kernels",
                                "achieved": round(achieved, 3), "peak": round(peak.value, 2), "unit": "TFLOP/s",
                                "frac": round(achieved / peak.value, 4), "ms": round(pair_ms, 5),
                                "algorithmic_flops": int(flops), "pairs_lj": n_lj, "pairs_coulomb": n_c},
        "roofline_spme": {
            "spread": hbm_roofline(spread_bytes, stages["spme_spread"], hbm, "k_bin_sites + k_spread_brick"),
            "gather": hbm_roofline(gather_bytes, stages["spme_gather"], hbm, "k_gather_brick + k_gather_wfin + k_recip_pass"),
            "stage": hbm_roofline(pme_bytes, pme_ms, hbm, "whole SPME stage incl. cuFFT"),
            "note": "algorithmic bytes: spread N_q*16 + K^3*4, gather N_q*16 + K^3*4 + N_q*12; the grid stays "
                    "in L2, so GB/s below HBM peak is expected"},
        "stage_ms": {k: round(v, 5) for k, v in stages.items()},
        "e2e": {"value": round(e2e_value, 2), "unit": "ns/day",
                "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes + 256},
        "gpu_launches": int(round(launches)),
        "clocks": clk,
        "cpu_baseline": cpu,
        "energies": {"temperature": round(en["temperature"], 2), "pressure_bar": round(en["pressure_bar"], 1),
                     "list_rebuilds": en["list_rebuilds"], "list_union_max": en["list_union_max"]},
        "wall_s": round(t_wall, 3),
    }
    if world == 1 and not args.no_extras and name in ("c3", "c3w"):
        # the headline metric covers the batched and served forms beside the
        # plain one: the c4 batch (64 members with peptides) and a c5-style
        # stream (400 requests of 1,000 steps; the c5 workload runs 5,000)
        try:
            b = measure_batch("c4", args, stream, dev)
            out["batched"] = b
            cap = b["member_steps_per_s"] / 1000.0
            out["served"] = measure_served("c5", args, stream.cuda_stream, capacity_req_per_s=cap)
        except Exception as e:  # reported, never fatal for the plain number
            out["batched_or_served_error"] = f"{type(e).__name__}: {e}"[:300]
    print(json.dumps(out))
    if dist:
        dist.destroy_process_group()


def profile_record(name):
    """The ncu summary numbers committed under profiles/ for this workload:
    {kernel: {dram_bytes_per_launch, ...}, "_source": file, "_captured": date}
    (profiles/traffic_<workload>.json), or {}."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", f"traffic_{name}.json")))
    except Exception:
        return {}


def roofline_dominant(name, flops, ms, peak, pc):
    """FP32 roofline of the water-water pair kernel: algorithmic FLOPs of the
    water-water site pairs inside the cutoff (19 + 15 per LJ pair, 19 + 23 per
    Coulomb pair, each pair once) per launch over its event-timed duration;
    traffic from the committed ncu capture of the same kernel."""
    rec = profile_record(name)
    k = rec.get("k_pair_ww_tile", {})
    return {"bound": "fp32", "kernel": "k_pair_ww_tile (water-water pairs)",
            "achieved": round(flops / (ms * 1e-3) / 1e12, 3), "peak": round(peak, 2), "unit": "TFLOP/s",
            "frac": round(flops / (ms * 1e-3) / 1e12 / peak, 4), "ms": round(ms, 5),
            "traffic": k.get("dram_bytes_per_launch"),
            "traffic_source": f"profiles/traffic_{name}.json ({rec.get('_captured', 'not captured')})",
            "peak_source": "measured FP32 FMA probe (dyn_probe_fp32_peak); MEASURED_PEAKS.json has no FP32 figure",
            "algorithmic_flops": int(flops), "pairs_lj_ww": pc["lj_ww"], "pairs_coulomb_ww": pc["coulomb_ww"]}


def hbm_roofline(nbytes, ms, peak, kernels):
    if not ms or ms <= 0:
        return None
    gbs = nbytes / (ms * 1e-3) / 1e9
    return {"bound": "hbm", "kernels": kernels, "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
            "frac": round(gbs / peak, 4) if peak else None, "ms": round(ms, 5), "algorithmic_bytes": int(nbytes)}


def cpu_baseline(name, args, sysd=None):
    """The C++ restatement of the reference CPU path on a bounded sample of
    the same system."""
    try:
        from oracle import cpu_ref
    except ImportError:
        return None
    try:
        return cpu_ref.run_sample(WORKLOADS[name], name, seconds=args.cpu_seconds, sysd=sysd)
    except Exception as e:  # the baseline is reported, never required
        return {"error": str(e)[:200]}


def run_reference_members(args, name):
    """Reference arm of the batched and serving workloads: the CPU
    restatement steps every member system one after another (the reference
    advances one MdState per call), each on a bounded sample."""
    from oracle import cpu_ref
    w = WORKLOADS[name]
    if w["kind"] == "batch":
        systems, _ = build_batch(name, seed=1)
        steps_each = 1
    else:
        from dynamics_b200 import synth
        sizes = synth.config4_sizes(w["n_req"], seed=7)
        systems = [synth.batch_member(int(n), seed=7000 + i)[0] for i, n in enumerate(sizes)]
        steps_each = w["steps_each"]
    per = max(0.5, args.cpu_seconds / len(systems))
    sec_per_step = 0.0
    cores = None
    for i, sysd in enumerate(systems):
        box = float(sysd["box_hi"][0])
        from dynamics_b200 import synth
        k = synth.fft_size(int(np.ceil(box)))
        wl = dict(n_water=len(sysd["water_pos"]), box=box, cutoff=w["cutoff"], grid=(k, k, k),
                  integrator=w["integrator"])
        res = cpu_ref.run_sample(wl, f"{name}[{i}]", seconds=per, steps=100000, warmup=1, sysd=sysd)
        sec_per_step += DT * 1e-3 * 86400.0 / res["value"]   # seconds per step of this member
        cores = res["cores"]
    value = len(systems) * DT * 1e-3 / sec_per_step * 86400.0
    cpu = {"value": round(value, 4), "unit": "ns/day (aggregate)", "cores": cores, "kind": "port",
           "sample": f"each of {len(systems)} members timed alone for ~{per:.1f} s, stepped one after another"}
    out = {"impl": "reference", "metric": "ns/day", "value": cpu["value"], "unit": cpu["unit"],
           "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps, "warmup": args.warmup,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic", "config": {"workload": name, "members": len(systems),
                                           "steps_each": steps_each},
           "cpu_baseline": cpu,
           "e2e": {"value": cpu["value"], "unit": cpu["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import cpu_ref
    name = args.workload
    if WORKLOADS[name].get("kind") in ("batch", "serve"):
        run_reference_members(args, name)
        return
    sysd, cfg = build_system(name, seed=1000)
    res = cpu_ref.run_sample(WORKLOADS[name], name, seconds=args.cpu_seconds, steps=args.steps,
                             warmup=args.warmup, sysd=sysd)
    out = {"impl": "reference", "metric": "ns/day", "value": res["value"], "unit": "ns/day",
           "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": res.get("steps"),
           "warmup": res.get("warmup"), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": plain_config(name, cfg, len(sysd["water_pos"]), len(sysd["atom_pos"]),
                                  int(os.environ.get("WORLD_SIZE", "1"))),
           "cpu_baseline": res,
           "e2e": {"value": res["value"], "unit": "ns/day", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def write_tune_table(path, names, steps=100, warmup=20):
    """Tunes every size class of the given workloads on this GPU (the
    autotuner timing whole captured steps, dynamics_b200.tune) and writes
    the table that dynamics_b200 ships as data/tune_b200.json: per class the
    chosen knobs and the milliseconds per step of every candidate."""
    import torch
    from dynamics_b200 import md, tune
    torch.cuda.set_device(0)
    os.environ["DYNB200_TUNE_CACHE"] = os.path.abspath(path)
    tune.SHIPPED = os.path.abspath(path) + ".none"  # tune everything here
    seen = set()
    for name in names:
        if WORKLOADS[name].get("kind") in ("batch", "serve"):
            systems, cfgs = build_batch(name, seed=1)
        else:
            s, c = build_system(name, 1)
            systems, cfgs = [s], [c]
        for sd, c in zip(systems, cfgs):
            key = tune.size_class(sd, c)
            if key in seen:
                continue
            seen.add(key)
            sd = md.equilibrate(sd, c, n_steps=200, dt=0.001)
            t0 = time.perf_counter()
            knobs = tune.tune(sd, c, steps=steps, warmup=warmup)
            print(json.dumps({"workload": name, "class": key, "knobs": knobs,
                              "s": round(time.perf_counter() - t0, 1)}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--equil", type=int, default=1000)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--tune", action="store_true",
                    help="batched workloads: also time the members with the autotuner's choices")
    ap.add_argument("--no-extras", action="store_true",
                    help="plain line only (no batched / served sub-objects)")
    ap.add_argument("--write-tune-table", metavar="PATH",
                    help="tune every size class of --tune-workloads and write the table to PATH")
    ap.add_argument("--tune-workloads", default="c1,c2,c3,c4")
    ap.add_argument("--set", action="append", default=[], metavar="FIELD=VALUE",
                    help="set an MdConfig field (numeric) for every system of the workload")
    args = ap.parse_args()
    for kv in args.set:
        k, _, val = kv.partition("=")
        CFG_OVERRIDES[k.strip()] = float(val) if "." in val else int(val)
    if args.write_tune_table:
        write_tune_table(args.write_tune_table, args.tune_workloads.split(","))
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif WORKLOADS[args.workload].get("kind") == "batch":
        run_batch(args)
    elif WORKLOADS[args.workload].get("kind") == "serve":
        run_serve(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
