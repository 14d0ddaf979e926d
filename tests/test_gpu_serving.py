"""Serving loop: requests of different physics, sizes and precisions, admitted as slots
and memory free up and stepped together, each give exactly the result they give alone.
Needs a B200."""
import numpy as np
import pytest

import lssph
from lssph import Request, Server

pytestmark = pytest.mark.gpu

MX = lssph.PRECISION_MIXED


def _requests():
    mk = [
        (lssph.make_params(lssph.taylor_green_params(num=48), precision=MX), 30),
        (lssph.cavity_params(num=40), 45),
        (lssph.make_params(lssph.boussinesq_params(num=40, ra=2e5), precision=MX), 25),
        (lssph.diffusion_params(num=30, seed=3), 40),
        (lssph.taylor_green_params(num=32, coe_cfl=0.2), 12),
        (lssph.make_params(lssph.cavity_params(num=32, re=400.0), precision=MX), 33),
        (lssph.make_params(lssph.boussinesq_params(num=32, ra=1e4), precision=MX), 19),
    ]
    return [Request(rid=i, params=p, nsteps=n) for i, (p, n) in enumerate(mk)]


def _solo(req):
    sim = lssph.Simulation.new(req.params)
    sim.step(req.nsteps)
    return sim.download()


def _fields(p):
    return ("x", "y", "u", "v", "rho", "pre") + (("tem",) if p.target_problem == 4 else ())


def test_each_result_is_the_same_alone_and_in_the_mix():
    reqs = _requests()
    srv = Server(max_active=3, chunk_steps=7)   # slots force queueing and staggered joins
    stats = srv.run(reqs, realtime=False)
    assert stats.completed == len(reqs)
    assert srv.peak_active == 3 and stats.batch_calls > 5
    for r in srv.done:
        assert r.stopped == "budget" and r.steps_done == r.nsteps and r.status == 0
        ref = _solo(r)
        for k in _fields(r.params):
            assert np.array_equal(getattr(r.result, k), getattr(ref, k)), (r.rid, k)
    srv.close()


def test_admission_by_hbm_footprint():
    reqs = _requests()
    big = max(lssph.estimate_device_bytes(r.params) for r in reqs)
    budget = int(1.5 * big)
    srv = Server(hbm_budget=budget, max_active=64, chunk_steps=10, keep_results=False)
    stats = srv.run(reqs, realtime=False)
    assert stats.completed == len(reqs)
    assert srv.peak_used <= budget
    assert srv.peak_active < len(reqs)          # memory, not slots, limited the mix
    with pytest.raises(ValueError):
        srv.submit(Request(rid=99, params=lssph.taylor_green_params(num=256), nsteps=1))
    srv.close()


def test_realtime_arrivals_report_latency():
    reqs = _requests()
    for i, r in enumerate(reqs):
        r.arrival = 0.02 * i
    srv = Server(max_active=8, chunk_steps=5, keep_results=False)
    stats = srv.run(reqs)
    assert stats.completed == len(reqs)
    assert all(r.admitted >= r.arrival for r in srv.done)
    assert 0 < stats.p50_s <= stats.p99_s
    assert stats.solves_per_s > 0 and stats.particle_updates_per_s > 0
    srv.close()


def test_preempted_requests_end_with_their_solo_result():
    # two long low-priority solves hold both slots; an urgent request arrives later and
    # suspends one of them (checkpoint to host), which later resumes from that checkpoint
    low = [Request(rid=0, params=lssph.taylor_green_params(num=48), nsteps=1500, arrival=0.0),
           Request(rid=1, params=lssph.cavity_params(num=48), nsteps=1500, arrival=0.0)]
    urgent = Request(rid=2, params=lssph.boussinesq_params(num=40), nsteps=60, arrival=0.03, priority=5)
    srv = Server(max_active=2, chunk_steps=20)
    stats = srv.run(low + [urgent], realtime=True)
    assert stats.completed == 3 and stats.preemptions >= 1
    assert any(r.preemptions > 0 for r in srv.done if r.rid != 2)
    done = {r.rid: r for r in srv.done}
    assert done[2].finished < max(done[0].finished, done[1].finished)
    for r in srv.done:
        assert r.stopped == "budget" and r.steps_done == r.nsteps and r.status == 0
        ref = _solo(r)
        for k in _fields(r.params):
            assert np.array_equal(getattr(r.result, k), getattr(ref, k)), (r.rid, k)
    srv.close()


def test_no_preemption_among_equal_priorities():
    reqs = _requests()
    srv = Server(max_active=2, chunk_steps=5, keep_results=False)
    stats = srv.run(reqs, realtime=False)
    assert stats.completed == len(reqs) and stats.preemptions == 0
    srv.close()
