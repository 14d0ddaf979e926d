"""Periodic domain on the GPU against the oracle's periodic extension (needs a B200).

A periodic square has no ghost particles; cells wrap and a neighbour across the boundary
is seen at its position shifted by -+L, on the GPU (staged halo cells carry the shift) as
in the oracle (each neighbour cell carries it).  Positions wrap into (0, L] after every
update.  Tolerances as for the closed box: lanes = 1 bit-identical, lanes = 4 relative L2
1e-10.  A uniform drift is added to the Taylor-Green state so that particles cross the
periodic boundary during the runs.
"""
import numpy as np
import pytest

import lssph
import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "u", "v", "rho", "pre")


def _pair(p, lanes, drift=0.0, amp=0.1, seed=0):
    q = lssph.make_params(p, lanes=lanes)
    st, ni = lssph.setup_particles(q)
    assert st.num_total == ni
    rng = np.random.default_rng(seed)
    if q.target_problem != 1:
        st.x[:] += amp * q.dx * (2 * rng.random(ni) - 1)
        st.y[:] += amp * q.dx * (2 * rng.random(ni) - 1)
        st.u[:] += drift
        st.v[:] += 0.5 * drift
    sim = lssph.Simulation(q, st, ni)
    orc = O.Oracle(q, st, ni, ghost=False)
    return sim, orc


def _rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


CASES = {
    "diffusion": lambda **kw: lssph.diffusion_params(num=40, seed=4, PERIODIC=1, **kw),
    "taylor_green": lambda **kw: lssph.taylor_green_params(num=48, PERIODIC=1, **kw),
    "taylor_green_classical": lambda **kw: lssph.taylor_green_params(num=48, PERIODIC=1, SPH_MODEL=2, **kw),
    "taylor_green_q9": lambda **kw: lssph.taylor_green_params(num=48, PERIODIC=1, SPH_MODEL=4, **kw),
    "taylor_green_rk2_quintic": lambda **kw: lssph.make_params(
        lssph.taylor_green_params(num=40, PERIODIC=1, KERNEL_TYPE=2, **kw), RK=2),
}


@pytest.mark.parametrize("case", list(CASES))
def test_neighbour_sets_across_the_boundary(case):
    p = CASES[case]()
    sim, orc = _pair(p, lanes=4, amp=0.3, seed=1)
    off_g, idx_g = sim.neighbors(0)
    off_o, idx_o = orc.neighbors(0)
    assert np.array_equal(off_g, off_o) and np.array_equal(idx_g, idx_o)
    sim.close()


@pytest.mark.parametrize("case", list(CASES))
def test_steps_bit_exact_with_one_lane(case):
    p = CASES[case]()
    nsteps = 40 if p.target_problem == 1 else 12
    sim, orc = _pair(p, lanes=1, drift=2.0, seed=2)
    sim.step(nsteps)
    orc.run(nsteps)
    g, o = sim.download(), orc.get()
    for k in FIELDS:
        assert np.array_equal(getattr(g, k), o[k]), k
    sim.close()


@pytest.mark.parametrize("case", list(CASES))
def test_steps_rel_l2(case):
    p = CASES[case]()
    nsteps = 300 if p.target_problem == 1 else 60
    sim, orc = _pair(p, lanes=4, drift=2.0, seed=3)
    sim.step(nsteps)
    orc.run(nsteps)
    g, o = sim.download(), orc.get()
    for k in ("u",) if p.target_problem == 1 else ("u", "v", "pre"):
        assert _rel_l2(getattr(g, k), o[k]) <= 1e-10, k
    if p.target_problem != 1:
        x0 = lssph.setup_particles(lssph.make_params(p, lanes=4))[0].x
        assert (g.x > 0).all() and (g.x <= p.len_x).all()
        assert np.abs(g.x - x0).max() > 0.5 * p.len_x      # some particles wrapped
    sim.close()


def test_periodic_diffusion_matches_the_analytic_decay():
    # configuration 1 as the benchmark writes it: sin(2 pi x) sin(2 pi y) exp(-8 pi^2 t)
    p = lssph.diffusion_params(num=64, seed=0, PERIODIC=1)
    sim = lssph.Simulation.new(p, ghost=False)
    n = 200
    sim.step(n)
    g, ni = sim.download(), sim.num_int
    ex = np.sin(2 * np.pi * g.x[:ni]) * np.sin(2 * np.pi * g.y[:ni]) * np.exp(-8 * np.pi ** 2 * n * p.dt)
    assert _rel_l2(g.u[:ni], ex) < 5e-3
    sim.close()


def test_mixed_precision_periodic_within_bound():
    # FP32 pair phase with the periodic shift in the FP32 offsets; bound as for the box
    p = lssph.taylor_green_params(num=64, PERIODIC=1)
    out = {}
    for prec in (lssph.PRECISION_FP64, lssph.PRECISION_MIXED):
        q = lssph.make_params(p, precision=prec)
        st, ni = lssph.setup_particles(q)
        st.u[:] += 2.0                       # particles cross the boundary
        sim = lssph.Simulation(q, st, ni)
        sim.step(100)
        out[prec] = sim.download()
        sim.close()
    a, b = out[lssph.PRECISION_FP64], out[lssph.PRECISION_MIXED]
    for k in ("u", "v", "rho"):
        assert _rel_l2(getattr(b, k), getattr(a, k)) <= 1e-5, k
    assert (b.x > 0).all() and (b.x <= p.len_x).all()


def test_periodic_members_in_a_batch_equal_solo():
    # periodic members (no ghosts: one bookkeeping CTA in the batched ghost launch) beside
    # closed-box ones; each ends bit for bit as it does alone
    mk = [lambda: lssph.taylor_green_params(num=48, PERIODIC=1),
          lambda: lssph.diffusion_params(num=40, seed=2, PERIODIC=1),
          lambda: lssph.cavity_params(num=40),
          lambda: lssph.make_params(lssph.taylor_green_params(num=32, PERIODIC=1), precision=lssph.PRECISION_MIXED)]

    def make(f, i):
        # lanes fixed: with lanes = 0 a solo run picks 2 or 4 by timing at its first launch,
        # while a batch member that never ran alone keeps 4
        p = lssph.make_params(f(), lanes=4)
        st, ni = lssph.setup_particles(p)
        if p.target_problem == 2:
            st.u[:ni] += 1.0
        sim = lssph.Simulation(p, st, ni)
        sim.ghost()
        return sim

    solo = [make(f, i) for i, f in enumerate(mk)]
    mem = [make(f, i) for i, f in enumerate(mk)]
    b = lssph.Batch()
    for m in mem:
        b.add(m)
    b.step(25)
    for s in solo:
        s.step(25)
    for i, (s, m) in enumerate(zip(solo, mem)):
        gs, gm = s.download(), m.download()
        for k in FIELDS:
            assert np.array_equal(getattr(gs, k), getattr(gm, k)), (i, k)
    b.close()
    for x in solo + mem:
        x.close()
