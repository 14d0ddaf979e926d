"""Batched time loop: every member of a batch must compute exactly what it computes
alone (bit-identical state, ghost values and RHS), whatever the other members are, and
whenever it joined.  Needs a B200.
"""
import numpy as np
import pytest

import lssph

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "u", "v", "rho", "pre", "tem")


def _sim(p, amp=0.1, seed=0):
    st, ni = lssph.setup_particles(p)
    rng = np.random.default_rng(seed)
    if p.target_problem != 1:
        st.x[:ni] += amp * p.dx * (2 * rng.random(ni) - 1)
        st.y[:ni] += amp * p.dx * (2 * rng.random(ni) - 1)
    sim = lssph.Simulation(p, st, ni)
    sim.ghost()
    return sim


# Mixed kinds: problem 1 (RK2, no PST), 2, 3 (RK4 + PST), 4 (temperature), a second
# Taylor-Green of another size and time step, one bit-exact-order solve (lanes = 1) and
# an RK2 solve of problem 3.
MEMBERS = [
    lambda: lssph.diffusion_params(num=30, seed=1),
    lambda: lssph.taylor_green_params(num=48),
    lambda: lssph.cavity_params(num=40),
    lambda: lssph.boussinesq_params(num=40, ra=1e5),
    lambda: lssph.taylor_green_params(num=32, coe_cfl=0.2),
    lambda: lssph.make_params(lssph.taylor_green_params(num=32), lanes=1),
    lambda: lssph.make_params(lssph.cavity_params(num=32), RK=2),
]


def _same(a: lssph.Simulation, b: lssph.Simulation, tag=""):
    ga, gb = a.download(), b.download()
    for k in FIELDS:
        if k == "tem" and a.params.target_problem != 4:
            continue
        assert np.array_equal(getattr(ga, k), getattr(gb, k)), (tag, k)
    va, vb = a.virtual_markers(), b.virtual_markers()
    for k in ("u", "v", "pre"):
        assert np.array_equal(va[k], vb[k]), (tag, "vm", k)
    ra, rb = a.rhs(), b.rhs()
    for k in ra:
        if ra[k] is not None:
            assert np.array_equal(ra[k], rb[k]), (tag, "rhs", k)


def test_batch_equals_solo_bit_exact():
    solo = [_sim(f(), seed=i) for i, f in enumerate(MEMBERS)]
    mem = [_sim(f(), seed=i) for i, f in enumerate(MEMBERS)]
    with lssph.Batch() as b:
        for m in mem:
            b.add(m)
        for _ in range(2):          # two calls: both step parities and descriptor reuse
            status, steady, steps = b.step(3)
            assert (steps == 3).all()
            assert (status == 0).all() and (steady == 0).all()
        ms, launches = b.last_step_stats()
        assert ms > 0 and launches > 0
    for s in solo:
        s.step(6)
    for i, (s, m) in enumerate(zip(solo, mem)):
        _same(s, m, i)


def test_membership_changes_between_calls():
    fa, fb, fc = MEMBERS[1], MEMBERS[3], MEMBERS[0]
    a, b_, c = _sim(fa(), seed=1), _sim(fb(), seed=2), _sim(fc(), seed=3)
    ra, rb, rc = _sim(fa(), seed=1), _sim(fb(), seed=2), _sim(fc(), seed=3)
    with lssph.Batch() as bt:
        bt.add(a)
        bt.add(b_)
        bt.step(3)
        bt.add(c)                   # joins late, at another parity than a and b
        bt.step(2)
        bt.remove(a)
        bt.step(3)
        assert len(bt) == 2
    ra.step(5)
    rb.step(8)
    rc.step(5)
    _same(a, ra, "a")
    _same(b_, rb, "b")
    _same(c, rc, "c")


def test_member_stepped_alone_between_calls():
    a, b_ = _sim(MEMBERS[1](), seed=5), _sim(MEMBERS[2](), seed=6)
    ra, rb = _sim(MEMBERS[1](), seed=5), _sim(MEMBERS[2](), seed=6)
    with lssph.Batch() as bt:
        bt.add(a)
        bt.add(b_)
        bt.step(2)
        a.step(1)                   # the batch must notice the parity change
        bt.step(2)
    ra.step(5)
    rb.step(4)
    _same(a, ra, "a")
    _same(b_, rb, "b")


def test_steady_state_per_member():
    p = lssph.diffusion_params(num=20, seed=2, THRESHOLD=2.0e-6)
    ref = _sim(p)
    s_ref = ref.step(5000)
    assert s_ref > 0
    d, t = _sim(p), _sim(MEMBERS[4](), seed=7)
    rt = _sim(MEMBERS[4](), seed=7)
    with lssph.Batch() as bt:
        bt.add(d)
        bt.add(t)
        status, steady, steps = bt.step(s_ref + 7)
    assert (status == 0).all()
    assert steady[0] == s_ref and steady[1] == 0
    assert steps[0] == s_ref and steps[1] == s_ref + 7
    rt.step(s_ref + 7)
    _same(d, ref, "diffusion")     # frozen at its steady state while the other ran on
    _same(t, rt, "taylor_green")


def test_error_is_isolated_to_its_member():
    p = lssph.taylor_green_params(num=32)
    st, ni = lssph.setup_particles(p)
    st.u[10] = np.nan
    bad = lssph.Simulation(p, st, ni)
    bad.ghost()
    good, ref = _sim(MEMBERS[2](), seed=8), _sim(MEMBERS[2](), seed=8)
    with lssph.Batch() as bt:
        bt.add(bad)
        bt.add(good)
        status, _, _ = bt.step(3, raise_on_error=False)
        with pytest.raises(lssph.LssphError):
            bt.step(1)
    assert status[0] == lssph._abi.E_NONFINITE and status[1] == 0
    ref.step(4)
    _same(good, ref, "good")


def test_one_launch_per_phase_for_many_members():
    sims = [_sim(lssph.taylor_green_params(num=32), seed=i) for i in range(16)]
    one = _sim(lssph.taylor_green_params(num=32), seed=0)
    one.step(2)
    with lssph.Batch() as bt:
        for s in sims:
            bt.add(s)
        bt.step(2)
        _, launches = bt.last_step_stats()
    # 16 solves, the 10 kernels of one RK4 + PST step plus the step-counter advance
    assert launches == 2 * 11
    _same(sims[0], one, "member 0")


def test_destroyed_member_leaves_the_batch():
    a, b_ = _sim(MEMBERS[1](), seed=1), _sim(MEMBERS[4](), seed=2)
    rb = _sim(MEMBERS[4](), seed=2)
    bt = lssph.Batch()
    bt.add(a)
    bt.add(b_)
    bt.step(1)
    a.close()
    bt.members = [m for m in bt.members if m is not a]
    assert bt._lib.lssph_batch_size(bt._b) == 1
    bt.step(2)
    bt.close()
    rb.step(3)
    _same(b_, rb, "b")


def test_step_budget_alone():
    p = MEMBERS[2]()
    a, ref = _sim(p, seed=11), _sim(p, seed=11)
    a.set_step_budget(7)
    a.step(10)
    assert a.progress() == (7, "budget")
    ref.step(7)
    _same(a, ref, "stopped at the budget")
    a.step(5)                       # no-op once stopped
    _same(a, ref, "still stopped")
    a.set_step_budget(0)            # resume
    a.step(3)
    ref.step(3)
    assert a.progress() == (10, "running")
    _same(a, ref, "resumed")


def test_step_budgets_in_a_batch():
    mk = [MEMBERS[1], MEMBERS[2], MEMBERS[3], MEMBERS[0], MEMBERS[6]]
    budgets = [3, 5, 8, 4, 6]
    mem = [_sim(f(), seed=20 + i) for i, f in enumerate(mk)]
    ref = [_sim(f(), seed=20 + i) for i, f in enumerate(mk)]
    with lssph.Batch() as bt:
        for m, n in zip(mem, budgets):
            m.set_step_budget(n)
            bt.add(m)
        status, _, steps = bt.step(10)
        assert (status == 0).all()
        assert list(steps) == budgets
        mem[2].set_step_budget(2)   # two more for one member, the others stay stopped
        _, _, steps = bt.step(4)
        assert list(steps) == [0, 0, 2, 0, 0]
    for r, n in zip(ref, budgets):
        r.step(n)
    ref[2].step(2)
    for i, (m, r) in enumerate(zip(mem, ref)):
        _same(m, r, i)


@pytest.mark.parametrize("k", range(len(MEMBERS)))
def test_footprint_estimate_matches_allocation(k):
    p = MEMBERS[k]()
    sim = lssph.Simulation.new(p)
    assert sim.device_bytes() == lssph.estimate_device_bytes(p)
