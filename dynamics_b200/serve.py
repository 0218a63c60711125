"""Serving form: a continuous-batching request loop over the batched engine.

Requests are independent MD systems, each asking for a number of steps.
They arrive over time; the server admits them in arrival order while the
device-memory budget and the member limit allow, keeps every admitted
system's coordinates, velocities, lists and PME grids resident in HBM, and
advances all admitted systems together (one kernel launch per stage for all
of them, dyn_batch_*) in rounds of ``round_steps`` steps.  Between rounds,
finished requests leave (their final state and energies are copied out) and
waiting requests join, so new work starts while earlier work is still on the
GPU.  Each result equals the result of the same request run alone.

The reference has no serving layer (one MdState per process,
src/integrate.rs:72); this module is new.
"""
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import md


@dataclass
class Request:
    rid: int
    system: dict
    cfg: md.MdConfig
    n_steps: int
    arrival: float                    # seconds after the server starts
    admitted: Optional[float] = None
    completed: Optional[float] = None
    state: Optional[dict] = None
    energies: Optional[dict] = None
    n_water: int = 0

    def __post_init__(self):
        self.n_water = len(np.asarray(self.system.get("water_pos", np.zeros((0, 3, 3)))).reshape(-1, 9))


@dataclass
class Report:
    requests: list
    wall_s: float
    steps_total: int
    dt_ps: float
    peak_members: int
    peak_bytes: int
    rounds: int
    budget_waits: int = 0             # admission points where the budget held a request back
    latency_s: dict = field(default_factory=dict)
    queue_wait_s: dict = field(default_factory=dict)

    @property
    def ns_per_day(self):
        return self.steps_total * self.dt_ps * 1e-3 / self.wall_s * 86400.0


def _pct(xs, q):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else float("nan")


class Server:
    """Continuous-batching server on one GPU.

    budget_bytes: device memory the admitted systems may hold together.
    max_members: most systems in flight at once.
    round_steps: steps between admission points; every request's step count
    and the SPME and energy intervals must divide it, so that each member's
    schedule is the one it has alone.
    """

    def __init__(self, budget_bytes=150e9, max_members=256, round_steps=100, dt=0.002, stream=None,
                 keep_states=True, clock=time.perf_counter):
        self.budget = float(budget_bytes)
        self.max_members = int(max_members)
        self.round_steps = int(round_steps)
        self.dt = float(dt)
        self.stream = stream
        self.keep_states = keep_states
        self.clock = clock
        self._bytes_per_water = None

    def _estimate(self, req):
        """Device bytes a request will hold: the largest per-water cost seen
        so far (a fresh server assumes 40 KB per water) plus its PME grid."""
        k = np.prod(req.cfg.spme_grid)
        per_water = self._bytes_per_water or 40e3
        return per_water * max(req.n_water, 1) + 16.0 * k + 8e6

    def run(self, requests):
        rs = self.round_steps
        for r in requests:
            if r.n_steps % rs:
                raise ValueError(f"request {r.rid}: n_steps must be a multiple of round_steps={rs}")
            if rs % max(1, r.cfg.spme_interval) or rs % max(1, r.cfg.energy_interval):
                raise ValueError("round_steps must be a multiple of the SPME and energy intervals")
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        batch = md.MdBatch(stream=self.stream)
        active = []        # [request, member, steps done, bytes]
        used = 0.0
        peak_members = 0
        peak_bytes = 0
        rounds = 0
        steps_total = 0
        budget_waits = 0
        t0 = self.clock()
        try:
            while pending or active:
                now = self.clock() - t0
                while pending and pending[0].arrival <= now and len(active) < self.max_members:
                    req = pending[0]
                    est = self._estimate(req)
                    if active and used + est > self.budget:
                        budget_waits += 1
                        break
                    pending.pop(0)
                    m = batch.add(req.system, req.cfg)
                    req.admitted = self.clock() - t0
                    nbytes = m.memory()
                    grid = 16.0 * np.prod(req.cfg.spme_grid)
                    bpw = max(0.0, nbytes - grid) / max(req.n_water, 1)
                    self._bytes_per_water = max(self._bytes_per_water or 0.0, bpw * 1.05)
                    used += nbytes
                    active.append([req, m, 0, nbytes])
                peak_members = max(peak_members, len(active))
                peak_bytes = max(peak_bytes, int(used))
                if not active:
                    wait = pending[0].arrival - (self.clock() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.05))
                    continue
                batch.step(self.dt, rs)
                batch.sync()
                rounds += 1
                steps_total += rs * len(active)
                still = []
                for a in active:
                    a[2] += rs
                    req, m = a[0], a[1]
                    if a[2] >= req.n_steps:
                        req.energies = m.energies()
                        if self.keep_states:
                            req.state = m.state()
                        req.completed = self.clock() - t0
                        batch.remove(m)
                        used -= a[3]
                    else:
                        still.append(a)
                active = still
        finally:
            batch.close()
        wall = self.clock() - t0
        lat = [r.completed - r.arrival for r in requests]
        wait = [r.admitted - r.arrival for r in requests]
        rep = Report(requests=list(requests), wall_s=wall, steps_total=steps_total, dt_ps=self.dt,
                     peak_members=peak_members, peak_bytes=peak_bytes, rounds=rounds, budget_waits=budget_waits)
        rep.latency_s = {"p50": _pct(lat, 50), "p99": _pct(lat, 99), "mean": float(np.mean(lat))}
        rep.queue_wait_s = {"p50": _pct(wait, 50), "p99": _pct(wait, 99), "mean": float(np.mean(wait))}
        return rep


def poisson_arrivals(n, rate_per_s, seed=0):
    """Arrival times of a seeded Poisson stream (exponential gaps)."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_per_s, n))
