"""The serving form (dynamics_b200.serve): requests that arrive while
others are on the GPU join the running batch between rounds; every result
must equal the same request run alone (bit-identical state and energies)."""
import numpy as np
import pytest

from dynamics_b200 import md, serve

from .test_gpu_batch import _members

pytestmark = pytest.mark.gpu


def _requests():
    systems, cfgs = _members()
    arrivals = [0.0, 0.0, 0.001, 0.002, 0.003]
    n_steps = [100, 50, 100, 150, 50]
    return [serve.Request(rid=i, system=s, cfg=c, n_steps=n, arrival=t)
            for i, (s, c, n, t) in enumerate(zip(systems, cfgs, n_steps, arrivals))]


def _alone(req):
    st = md.MdState(req.system, req.cfg)
    st.step(0.002, req.n_steps)
    out = st.state(), st.energies()
    st.close()
    return out


def test_served_results_equal_alone(gpu_lib):
    reqs = _requests()
    # at most two in flight: the later requests wait, then join a running batch
    rep = serve.Server(round_steps=50, max_members=2).run(reqs)
    assert rep.peak_members == 2
    assert all(r.completed is not None for r in reqs)
    joined_late = [r for r in reqs if r.admitted > min(q.admitted for q in reqs) and r.rid >= 2]
    assert joined_late, "no request joined while others were running"
    for r in reqs:
        st, en = _alone(r)
        for k in st:
            np.testing.assert_array_equal(st[k], r.state[k], err_msg=f"request {r.rid} {k}")
        for k in ("potential", "kinetic", "virial", "temperature", "step"):
            assert en[k] == r.energies[k], (r.rid, k, en[k], r.energies[k])
    assert np.isfinite(rep.latency_s["p99"]) and rep.latency_s["p99"] >= rep.latency_s["p50"] > 0
    assert rep.queue_wait_s["p99"] > 0
    assert rep.steps_total == sum(r.n_steps for r in reqs)


def test_budget_limits_admission(gpu_lib):
    reqs = _requests()
    # a budget below two systems' footprint: one request at a time
    rep = serve.Server(budget_bytes=1.0, round_steps=50).run(reqs)
    assert rep.peak_members == 1
    assert all(r.completed is not None for r in reqs)


def test_rejects_misaligned_steps(gpu_lib):
    reqs = _requests()
    reqs[0].n_steps = 75
    with pytest.raises(ValueError):
        serve.Server(round_steps=50).run(reqs)
