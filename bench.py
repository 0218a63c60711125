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
    "c5w": dict(kind="serve", n_req=48, rate=20.0, steps_each=5000, cutoff=9.0, budget=150e9,
                integrator="langevin", barostat=False, n_water=None),
    # as c4w / c5w with 0-3 ten-residue ff19SB peptides (and counter-ions,
    # bond-to-H constraints) in every member
    "c4": dict(kind="batch", n_sys=64, cutoff=9.0, integrator="langevin", barostat=False,
               n_water=None, peptides=3),
    "c5": dict(kind="serve", n_req=48, rate=20.0, steps_each=5000, cutoff=9.0, budget=150e9,
               integrator="langevin", barostat=False, n_water=None, peptides=3),
}
DEFAULT_WORKLOAD = "c3"
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one step's
# short-range pair kernels (water-water, water-atom, atom-atom), from an
# ncu --set full capture of the workload (cold L2, as in the timed loop,
# which flushes L2 between steps)
PAIR_DRAM_BYTES = {"c3w": 17306880, "c3": 17521920 + 4856576 + 905984}
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
    return sysd, cfg


def member_system(w, n_water, seed, rng):
    """One batched / served member: a water box, or with w["peptides"] a box
    with 0..w["peptides"] ten-residue peptides (count drawn from rng)."""
    from dynamics_b200 import synth
    if w.get("peptides"):
        from dynamics_b200 import peptide
        n_pep = int(rng.integers(0, w["peptides"] + 1))
        sysd, grid, _ = peptide.batch_member(int(n_water), n_pep, seed=seed)
        return sysd, grid
    return synth.batch_member(int(n_water), seed=seed)


def build_batch(name, seed):
    from dynamics_b200 import md, synth
    w = WORKLOADS[name]
    sizes = synth.config4_sizes(w["n_sys"], seed=seed)
    rng = np.random.default_rng(seed + 7919)
    systems, cfgs = [], []
    alpha = synth.ewald_alpha(w["cutoff"])
    for i, n in enumerate(sizes):
        sysd, grid = member_system(w, n, seed * 1000 + i, rng)
        cfg = md.MdConfig(coulomb_cutoff=w["cutoff"], lj_cutoff=w["cutoff"], spme_alpha=alpha,
                          spme_grid=grid, seed=seed * 1000 + i,
                          integrator=md.LangevinMiddle(gamma=1.0))
        systems.append(sysd)
        cfgs.append(cfg)
    return systems, cfgs


def run_batch(args):
    """Batched form: aggregate ns/day of all members advanced together,
    against the same systems stepped one by one through the plain path."""
    import torch

    from dynamics_b200 import md
    rank, world, local, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    name = args.workload
    w = WORKLOADS[name]
    systems, cfgs = build_batch(name, seed=1 + rank)
    systems = [md.equilibrate(s, c, n_steps=min(args.equil, 200), dt=0.001) for s, c in zip(systems, cfgs)]
    n_sys = len(systems)
    n_water = int(sum(len(s["water_pos"]) for s in systems))
    n_atoms = int(sum(len(s.get("atom_pos", ())) for s in systems))
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    # ---- plain path, one system at a time (each its own graph per step) ----
    k_plain = max(10, min(args.steps, 100))
    plain_ms = 0.0
    for s, c in zip(systems, cfgs):
        st = md.MdState(s, c, stream=stream.cuda_stream)
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
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(clock_csv(rank))
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with clocks:
        for k in range(args.steps):
            flush.zero_()
            ev0[k].record(stream)
            batch.step(DT, 1)
            ev1[k].record(stream)
        torch.cuda.synchronize(dev)
    batch.sync()
    ms = max_over_ranks(float(np.sum([ev0[k].elapsed_time(ev1[k]) for k in range(args.steps)])), dist, dev)
    rebuilds = sum(m.energies()["list_rebuilds"] for m in batch.members) - r0
    fixed_s, reb_k, per_k = batch.launches(True)
    fixed_n, _, _ = batch.launches(False)
    launches = (fixed_s + fixed_n) / 2.0 * args.steps + reb_k * min(rebuilds, args.steps)
    value = aggregate_ns_per_day(args.steps, n_sys, world, ms)
    plain_value = DT * 1e-3 * n_sys / (plain_ms * 1e-3) * 86400.0
    # ---- end to end: every member's positions/velocities in and out per step ----
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).pin_memory().numpy()
    keys = ("water_pos", "water_vel", "atom_pos", "atom_vel")
    host = []
    for m in batch.members:
        s0 = m.state()
        host.append({k: pin(s0[k]) for k in keys if k in s0 and s0[k].size})
    n_e2e = max(5, args.steps // 20)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        for m, hb in zip(batch.members, host):
            m.set_state(**hb)
        batch.step(DT, 1)
        for m, hb in zip(batch.members, host):
            s1 = m.state()
            for k in hb:
                hb[k][:] = s1[k]
    t_e2e = time.perf_counter() - t0
    e2e_value = n_e2e * DT * 1e-3 * n_sys * world / t_e2e * 86400.0
    io_bytes = int(sum(a.nbytes for hb in host for a in hb.values()))
    clk = clocks.summary(local)
    batch.close()
    if dist:
        dist.barrier()
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    out = {
        "metric": "ns/day", "value": round(value, 2), "unit": "ns/day (aggregate over members)",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 5), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded OPC water boxes" + (", 0-3 ten-residue ff19SB peptides each"
                                                        if w.get("peptides") else "")
                + ", equilibrated on device)",
        "config": {"workload": name, "members": n_sys, "n_water_total": n_water,
                   "n_atoms_total": n_atoms, "sizes": "512-8000 waters, log-uniform", "cutoff_A": w["cutoff"],
                   "grid": "FFT-friendly ~1 A", "integrator": "langevin_middle", "dt_fs": DT * 1e3,
                   "l2": "256 MiB flush between timed steps", "parallelism": f"replicas x{world}"},
        "plain_one_by_one": {"value": round(plain_value, 2), "unit": "ns/day (aggregate)",
                             "ms_per_round": round(plain_ms, 4), "steps_each": k_plain,
                             "batch_over_plain": round(value / world / plain_value, 3)},
        "e2e": {"value": round(e2e_value, 2), "unit": "ns/day (aggregate)",
                "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes},
        "gpu_launches": int(round(launches)),
        "launches_per_step": {"spme": fixed_s, "no_spme": fixed_n, "rebuild_extra": reb_k,
                              "periodic_extra": per_k},
        "clocks": clk, "cpu_baseline": None,
    }
    print(json.dumps(out))
    if dist:
        dist.destroy_process_group()


def run_serve(args):
    """Serving form: p50/p99 completion latency, queue wait and aggregate
    ns/day of a continuous-batching server, against the same requests served
    one at a time through the plain path (first come, first served)."""
    import torch

    from dynamics_b200 import md, serve, synth
    rank, world, local, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    name = args.workload
    w = WORKLOADS[name]
    seed = 7 + rank
    sizes = synth.config4_sizes(w["n_req"], seed=seed)
    arrivals = serve.poisson_arrivals(w["n_req"], w["rate"], seed=seed)
    alpha = synth.ewald_alpha(w["cutoff"])
    reqs = []
    rng = np.random.default_rng(seed + 7919)
    for i, (n, t) in enumerate(zip(sizes, arrivals)):
        sysd, grid = member_system(w, n, seed * 1000 + i, rng)
        cfg = md.MdConfig(coulomb_cutoff=w["cutoff"], lj_cutoff=w["cutoff"], spme_alpha=alpha, spme_grid=grid,
                          seed=seed * 1000 + i, integrator=md.LangevinMiddle(gamma=1.0))
        sysd = md.equilibrate(sysd, cfg, n_steps=min(args.equil, 200), dt=0.001)
        reqs.append(serve.Request(rid=i, system=sysd, cfg=cfg, n_steps=w["steps_each"], arrival=float(t)))
    # plain path, one request at a time: time each alone on a bounded sample
    k_plain = max(20, min(args.steps, 500))
    per_step = []
    for r in reqs:
        st = md.MdState(r.system, r.cfg, stream=stream.cuda_stream)
        st.step(DT, args.warmup)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        st.step(DT, k_plain)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        per_step.append(e0.elapsed_time(e1) / k_plain * 1e-3)
        st.close()
    done = 0.0
    lat_plain = []
    for r, t in zip(reqs, per_step):
        done = max(done, r.arrival) + t * r.n_steps
        lat_plain.append(done - r.arrival)
    plain_ns_day = sum(r.n_steps for r in reqs) * DT * 1e-3 / done * 86400.0
    clocks = ClockSampler(clock_csv(rank))
    srv = serve.Server(budget_bytes=w["budget"], round_steps=100, dt=DT, stream=stream.cuda_stream,
                       keep_states=False)
    if dist:
        dist.barrier()
    with clocks:
        rep = srv.run(reqs)
    clk = clocks.summary(local)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    io = int(sum(r.system["water_pos"].nbytes + r.system["water_vel"].nbytes for r in reqs))
    out = {
        "metric": "ns/day", "value": round(rep.ns_per_day, 2), "unit": "ns/day (aggregate over requests)",
        "n_gpus": world, "steps": rep.steps_total, "warmup": args.warmup,
        "ms_per_step": round(rep.wall_s / rep.rounds / 100 * 1e3, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded OPC water boxes" + (", 0-3 ten-residue ff19SB peptides each"
                                                        if w.get("peptides") else "")
                + ", equilibrated on device before arrival)",
        "config": {"workload": name, "requests": len(reqs), "arrival_rate_per_s": w["rate"],
                   "steps_each": w["steps_each"], "sizes": "512-8000 waters, log-uniform",
                   "budget_GB": w["budget"] / 1e9, "round_steps": 100, "integrator": "langevin_middle",
                   "dt_fs": DT * 1e3, "parallelism": f"replicas x{world}"},
        "latency_s": {k: round(v, 4) for k, v in rep.latency_s.items()},
        "queue_wait_s": {k: round(v, 4) for k, v in rep.queue_wait_s.items()},
        "wall_s": round(rep.wall_s, 3), "peak_members": rep.peak_members,
        "peak_device_GB": round(rep.peak_bytes / 1e9, 3),
        "plain_one_at_a_time": {
            "value": round(plain_ns_day, 2), "unit": "ns/day (aggregate)",
            "latency_s": {"p50": round(float(np.percentile(lat_plain, 50)), 4),
                          "p99": round(float(np.percentile(lat_plain, 99)), 4)},
            "note": f"each request timed alone over {k_plain} steps and scaled to its step count, "
                    "served first come first served"},
        "e2e": {"value": round(rep.ns_per_day, 2), "unit": "ns/day (aggregate)", "h2d_bytes_per_step": None,
                "d2h_bytes_per_step": None,
                "note": f"inputs ({io} bytes in total) enter through the public API at admission and results "
                        "leave at completion, inside the timed region"},
        "clocks": clk, "cpu_baseline": None,
    }
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
        t = cKDTree(np.mod(pts - lo, ext), boxsize=ext)
        p = t.query_pairs(cutoff, output_type="ndarray")
        keep = mol[p[:, 0]] != mol[p[:, 1]]
        p = p[keep]
        if excl:
            a, b = atom_id[p[:, 0]], atom_id[p[:, 1]]
            both = (a >= 0) & (b >= 0)
            if both.any():
                pa = np.sort(np.stack([a[both], b[both]], 1), axis=1)
                ex = np.array([tuple(x) in excl for x in pa.tolist()])
                return int(len(p) - np.count_nonzero(ex))
        return int(len(p))

    ljm = np.asarray(sysd.get("atom_eps", np.zeros(na))) > 0
    qm = np.asarray(sysd.get("atom_q", np.zeros(na))) != 0
    amol = -1 - np.arange(na)
    aid = np.arange(na)
    lj_pts = np.concatenate([o, ap[ljm]])
    lj_mol = np.concatenate([np.arange(nw), amol[ljm]])
    lj_id = np.concatenate([np.full(nw, -1), aid[ljm]])
    n_lj = npairs(lj_pts, lj_mol, lj_id)
    q_pts = np.concatenate([wp[:, 1], wp[:, 2], m, ap[qm]])
    q_mol = np.concatenate([np.tile(np.arange(nw), 3), amol[qm]])
    q_id = np.concatenate([np.full(3 * nw, -1), aid[qm]])
    n_c = npairs(q_pts, q_mol, q_id)
    return n_lj, n_c


class ClockSampler:
    def __init__(self, path):
        self.path = path
        self.proc = None

    def __enter__(self):
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
    n_lj, n_c = count_pairs({**sysd, "water_pos": st.state()["water_pos"]}, w["cutoff"])
    flops = n_lj * (19 + 15) + n_c * (19 + 23)   # frozen per-pair convention
    pair_ms = stages["pairs"]
    achieved = flops / (pair_ms * 1e-3) / 1e12
    import ctypes as C
    peak = C.c_double()
    _lib.check(_lib.lib().dyn_probe_fp32_peak(stream.cuda_stream, C.byref(peak)))
    # PME: algorithmic bytes of spread + gather per SPME step
    nq = 3 * st.n_water + st.n_atoms
    K = np.prod(w["grid"])
    pme_bytes = nq * 16 + K * 4 + nq * 16 + K * 4 + nq * 12
    pme_ms = stages["spme"]
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
    launches = ((st.launches_per_step(True) + st.launches_per_step(False)) / 2.0 * args.steps
                + rebuilds * n_rebuild_k + due * n_periodic_k)
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
        "roofline": {"bound": "fp32", "kernel": "short-range pair kernels",
                     "achieved": round(achieved, 3), "peak": round(peak.value, 2), "unit": "TFLOP/s",
                     "frac": round(achieved / peak.value, 4), "traffic": PAIR_DRAM_BYTES.get(name),
                     "peak_source": "measured FP32 FMA probe (dyn_probe_fp32_peak)",
                     "algorithmic_flops": int(flops), "pairs_lj": n_lj, "pairs_coulomb": n_c},
        "roofline_spme": {"bound": "hbm", "achieved": round(pme_bytes / (pme_ms * 1e-3) / 1e9, 1),
                          "peak": hbm, "unit": "GB/s",
                          "frac": round(pme_bytes / (pme_ms * 1e-3) / 1e9 / hbm, 4) if hbm else None,
                          "note": "whole SPME stage incl. cuFFT; grid is L2-resident"},
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
    print(json.dumps(out))
    if dist:
        dist.destroy_process_group()


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
    args = ap.parse_args()
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
