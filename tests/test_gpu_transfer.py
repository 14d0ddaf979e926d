"""Host transfers through page-locked buffers (needs a B200).

lssph_upload and lssph_download read and write page-locked, mapped host buffers (from
cudaHostAlloc, or torch's pin_memory) directly from one kernel, and go through copies for
ordinary pageable memory.  Both paths must move the same bytes: a download fills the
same values, and a solve continues bit for bit from either upload.
"""
import numpy as np
import pytest
import torch

import lssph

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "u", "v", "rho", "pre")

CASES = {
    "diffusion": lambda: lssph.diffusion_params(num=40, seed=3),
    "taylor_green": lambda: lssph.taylor_green_params(num=48),
    # lanes fixed: with lanes = 0 each handle of a periodic solve picks 2 or 4 by timing
    "taylor_green_periodic": lambda: lssph.taylor_green_params(num=48, PERIODIC=1, lanes=4),
    "cavity": lambda: lssph.cavity_params(num=40),
    "boussinesq": lambda: lssph.boussinesq_params(num=40),
}


def _pinned(a):
    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy()
    t[:] = a
    return t


def _pinned_state(st, with_tem):
    tem = _pinned(st.tem) if with_tem else None
    return lssph.State(st.ptype.copy(), *(_pinned(getattr(st, k)) for k in FIELDS), tem)


def _sim(p):
    s = lssph.Simulation.new(p)
    return s


def _keys(p):
    return FIELDS + (("tem",) if p.target_problem == 4 else ())


@pytest.mark.parametrize("case", list(CASES))
def test_pinned_download_equals_pageable(case):
    p = CASES[case]()
    sim = _sim(p)
    sim.step(7)
    ref = sim.download()
    pin = _pinned_state(ref, p.target_problem == 4)
    for k in _keys(p):
        getattr(pin, k)[:] = -1.0
    sim.download_into(pin)
    for k in _keys(p):
        assert np.array_equal(getattr(pin, k), getattr(ref, k)), k
    sim.close()


@pytest.mark.parametrize("case", list(CASES))
def test_pinned_upload_mid_run_equals_pageable(case):
    p = CASES[case]()
    a, b, c = _sim(p), _sim(p), _sim(p)
    a.step(10)
    mid = a.download()
    a.step(10)
    b.step(3)                     # b and c are elsewhere in their runs
    b.upload(mid)
    b.step(10)
    c.step(3)
    c.upload(_pinned_state(mid, p.target_problem == 4))
    c.step(10)
    ga, gb, gc = a.download(), b.download(), c.download()
    for k in _keys(p):
        assert np.array_equal(getattr(gb, k), getattr(ga, k)), k
        assert np.array_equal(getattr(gc, k), getattr(ga, k)), k
    for s in (a, b, c):
        s.close()


def test_pinned_round_trip_every_step_equals_resident_run():
    # the end-to-end pattern: upload, one step, download, each step, from pinned buffers
    p = lssph.taylor_green_params(num=64, PERIODIC=1, lanes=4)
    res, e2e = _sim(p), _sim(p)
    host = _pinned_state(e2e.download(), False)
    for _ in range(12):
        e2e.upload(host)
        e2e.step(1)
        e2e.download_into(host)
    res.step(12)
    g = res.download()
    for k in FIELDS:
        assert np.array_equal(getattr(host, k), getattr(g, k)), k
    res.close()
    e2e.close()


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("case", list(CASES))
def test_advance_host_equals_upload_step_download(case, pinned):
    # lssph_advance_host (one call, one synchronisation) against the three separate calls,
    # every step from the host arrays, with page-locked and with pageable buffers
    p = CASES[case]()
    sep, fused = _sim(p), _sim(p)
    a = sep.download()
    b = _pinned_state(a, p.target_problem == 4) if pinned else sep.download()
    for n in (1, 3, 1):
        sep.upload(a)
        sep.step(n)
        sep.download_into(a)
        assert fused.advance_host(b, n) == 0
        for k in _keys(p):
            assert np.array_equal(getattr(b, k), getattr(a, k)), (n, k)
    sep.close()
    fused.close()


def test_advance_host_returns_the_state_where_a_stopped_solve_stopped():
    # a solve that stops part-way through the call (its step budget; problem 1: its steady
    # state) hands back the state of its last executed step, as step + download give it.
    # RK4 + PST flips the state buffers an odd number of times per step, so three of four
    # steps leave the other buffer current than four would.
    p = lssph.taylor_green_params(num=48)
    sep, fused = _sim(p), _sim(p)
    a = sep.download()
    b = _pinned_state(a, False)
    for s in (sep, fused):
        s.set_step_budget(3)
    sep.upload(a)
    sep.step(4)
    sep.download_into(a)
    fused.advance_host(b, 4)
    assert sep.progress() == fused.progress() == (3, "budget")
    for k in FIELDS:
        assert np.array_equal(getattr(b, k), getattr(a, k)), k
    q = lssph.diffusion_params(num=24, seed=1, THRESHOLD=1e-3)
    sep, fused = _sim(q), _sim(q)
    a = sep.download()
    b = _pinned_state(a, False)
    sep.upload(a)
    s1 = sep.step(800)
    sep.download_into(a)
    s2 = fused.advance_host(b, 800)
    assert 0 < s1 == s2 < 800
    for k in FIELDS:
        assert np.array_equal(getattr(b, k), getattr(a, k)), k
    sep.close()
    fused.close()
