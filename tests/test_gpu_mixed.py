"""Mixed precision: FP32 kernel weights, basis and neighbour sums (over FP64-formed,
FP32-rounded offsets and field differences), FP64 moment-matrix factorisation (the
compensated mode: Kahan-compensated sums and one refinement step of the solve), FP64 RK
update.

Bound (stated): every field within relative L2 1e-5 of the FP64 path on the same inputs
after the stated step count, and analytical-solution errors unchanged.  Needs a B200.
"""
import numpy as np
import pytest

import lssph
import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5
CASES = {
    "diffusion": (lambda: lssph.diffusion_params(num=50, seed=1), 1000),
    "taylor_green": (lambda: lssph.taylor_green_params(num=64), 400),
    "cavity": (lambda: lssph.cavity_params(num=64), 400),
    "boussinesq": (lambda: lssph.boussinesq_params(num=48, ra=1e5), 400),
}


def _fields(p):
    return ("x", "y", "u", "v", "rho", "pre") + (("tem",) if p.target_problem == 4 else ())


def _sim(p, precision, amp=0.1, seed=0):
    q = lssph.make_params(p, precision=precision)
    st, ni = lssph.setup_particles(q)
    rng = np.random.default_rng(seed)
    if q.target_problem != 1:
        st.x[:ni] += amp * q.dx * (2 * rng.random(ni) - 1)
        st.y[:ni] += amp * q.dx * (2 * rng.random(ni) - 1)
    sim = lssph.Simulation(q, st, ni)
    sim.ghost()
    return sim


def _rel(a, b):
    n = np.linalg.norm(b)
    return np.linalg.norm(a - b) / n if n > 0 else np.linalg.norm(a - b)


@pytest.mark.parametrize("prec", [lssph.PRECISION_MIXED, lssph.PRECISION_MIXED_COMPENSATED])
@pytest.mark.parametrize("case", list(CASES))
def test_mixed_within_bound_of_fp64(case, prec):
    # both mixed modes: plain FP32 lane sums and Kahan-compensated ones
    mk, steps = CASES[case]
    p = mk()
    s64 = _sim(p, lssph.PRECISION_FP64)
    smx = _sim(p, prec)
    assert s64.step(steps) == smx.step(steps) == 0
    g64, gmx = s64.download(), smx.download()
    ni = s64.num_int
    for k in _fields(p):
        err = _rel(getattr(gmx, k)[:ni], getattr(g64, k)[:ni])
        assert err <= TOL, (k, err)
    assert not np.array_equal(gmx.u, g64.u)   # it is a different arithmetic


def test_mixed_against_the_oracle():
    p = lssph.cavity_params(num=48)
    smx = _sim(p, lssph.PRECISION_MIXED, seed=3)
    st, ni = lssph.setup_particles(p)
    rng = np.random.default_rng(3)
    st.x[:ni] += 0.1 * p.dx * (2 * rng.random(ni) - 1)
    st.y[:ni] += 0.1 * p.dx * (2 * rng.random(ni) - 1)
    orc = O.Oracle(p, st, ni, ghost=True)
    smx.step(50)
    orc.run(50)
    g, o = smx.download(), orc.get()
    for k in _fields(p):
        assert _rel(getattr(g, k)[:ni], o[k][:ni]) <= TOL, k


def test_mixed_taylor_green_decay_error_unchanged():
    # velocity amplitude decays as exp(-8 pi^2 t / Re) (TG_A = TG_B = 2)
    p = lssph.taylor_green_params(num=64, re=100.0)
    errs = {}
    for prec in (lssph.PRECISION_FP64, lssph.PRECISION_MIXED):
        sim = _sim(p, prec, amp=0.0)
        u0 = sim.download()
        n = 800
        sim.step(n)
        g = sim.download()
        ni = sim.num_int
        decay = np.exp(-8.0 * np.pi ** 2 * (n * p.dt) / 100.0)
        ref = np.hypot(u0.u[:ni], u0.v[:ni]) * decay
        errs[prec] = np.linalg.norm(np.hypot(g.u[:ni], g.v[:ni]) - ref) / np.linalg.norm(ref)
    # the discretisation error dominates; mixed precision moves it by well under 1%
    assert abs(errs[lssph.PRECISION_MIXED] - errs[lssph.PRECISION_FP64]) <= 1e-2 * errs[lssph.PRECISION_FP64], errs


@pytest.mark.parametrize("case", ["taylor_green", "cavity", "boussinesq"])
def test_mixed_two_lanes_within_bound_of_fp64(case):
    # the mixed kernels at 2 lanes per particle: the same sums split over 2 lanes, the same
    # bound against FP64
    mk, steps = CASES[case]
    p = mk()
    s64 = _sim(p, lssph.PRECISION_FP64)
    smx = _sim(lssph.make_params(p, lanes=2), lssph.PRECISION_MIXED)
    assert smx.tuning()["lanes"] == 2
    assert s64.step(steps) == smx.step(steps) == 0
    g64, gmx = s64.download(), smx.download()
    ni = s64.num_int
    for k in _fields(p):
        err = _rel(getattr(gmx, k)[:ni], getattr(g64, k)[:ni])
        assert err <= TOL, (k, err)


def test_mixed_two_lane_members_identical_alone_and_batched():
    mk = [lambda: lssph.make_params(lssph.taylor_green_params(num=48, PERIODIC=1), lanes=2),
          lambda: lssph.make_params(lssph.cavity_params(num=40), lanes=2)]
    solo = [_sim(f(), lssph.PRECISION_MIXED, seed=i) for i, f in enumerate(mk)]
    mem = [_sim(f(), lssph.PRECISION_MIXED, seed=i) for i, f in enumerate(mk)]
    with lssph.Batch() as b:
        for m in mem:
            b.add(m)
        b.step(5)
    for s in solo:
        s.step(5)
    for s, m in zip(solo, mem):
        gs, gm = s.download(), m.download()
        for k in _fields(s.params):
            assert np.array_equal(getattr(gs, k), getattr(gm, k)), k


def test_mixed_members_identical_alone_and_batched():
    mk = [lambda: lssph.taylor_green_params(num=48), lambda: lssph.boussinesq_params(num=40),
          lambda: lssph.diffusion_params(num=30)]
    solo = [_sim(f(), lssph.PRECISION_MIXED, seed=i) for i, f in enumerate(mk)]
    mem = [_sim(f(), lssph.PRECISION_MIXED, seed=i) for i, f in enumerate(mk)]
    fp64 = _sim(lssph.cavity_params(num=32), lssph.PRECISION_FP64, seed=9)
    ref64 = _sim(lssph.cavity_params(num=32), lssph.PRECISION_FP64, seed=9)
    with lssph.Batch() as b:
        for m in mem + [fp64]:
            b.add(m)
        b.step(5)
    for s in solo + [ref64]:
        s.step(5)
    for s, m in zip(solo + [ref64], mem + [fp64]):
        gs, gm = s.download(), m.download()
        for k in _fields(s.params):
            assert np.array_equal(getattr(gs, k), getattr(gm, k)), k


def test_compensated_and_plain_mixed_members_identical_alone_and_batched():
    # a batch holding both mixed modes keeps them in separate groups; each member ends
    # bit for bit as it does alone
    mk = [(lambda: lssph.taylor_green_params(num=48), lssph.PRECISION_MIXED_COMPENSATED),
          (lambda: lssph.taylor_green_params(num=48), lssph.PRECISION_MIXED),
          (lambda: lssph.cavity_params(num=40), lssph.PRECISION_MIXED_COMPENSATED)]
    solo = [_sim(f(), prec, seed=i) for i, (f, prec) in enumerate(mk)]
    mem = [_sim(f(), prec, seed=i) for i, (f, prec) in enumerate(mk)]
    with lssph.Batch() as b:
        for m in mem:
            b.add(m)
        b.step(5)
    for s in solo:
        s.step(5)
    for s, m in zip(solo, mem):
        gs, gm = s.download(), m.download()
        for k in _fields(s.params):
            assert np.array_equal(getattr(gs, k), getattr(gm, k)), k
    # the two modes are different arithmetic on the same inputs
    assert not np.array_equal(solo[0].download().u, solo[1].download().u)


def test_split_precision_positions_follow_the_fp64_positions():
    # the FP32 offsets from the cell origins that the mixed staging reads: a mixed solve that
    # is downloaded, re-created from its state (which recomputes the offsets from the FP64
    # positions) and stepped on ends bit for bit as the uninterrupted solve
    p = lssph.make_params(lssph.cavity_params(num=40), lanes=4)
    a = _sim(p, lssph.PRECISION_MIXED, seed=5)
    b = _sim(p, lssph.PRECISION_MIXED, seed=5)
    a.step(7)
    b.step(4)
    c = lssph.Simulation(b.params, b.download(), b.num_int)
    c.step(3)
    ga, gc = a.download(), c.download()
    for k in _fields(p):
        assert np.array_equal(getattr(ga, k), getattr(gc, k)), k


@pytest.mark.parametrize("prec", [lssph.PRECISION_MIXED, lssph.PRECISION_MIXED_COMPENSATED])
@pytest.mark.parametrize("case", list(CASES))
def test_split_and_fused_shapes_give_identical_bits(case, prec, monkeypatch):
    # the split shape (pair kernel, then one solve-and-update thread per particle) runs the
    # fused kernels' arithmetic per particle: same bits, every field, stages and PST
    mk, _ = CASES[case]
    out = {}
    for shape in ("fused", "split"):
        monkeypatch.setenv("LSSPH_KERNEL_SHAPE", shape)
        sim = _sim(lssph.make_params(mk(), lanes=4), prec, seed=4)
        sim.step(6)
        assert sim.tuning()["shape"] == shape
        out[shape] = sim.download()
        sim.close()
    for k in _fields(mk()):
        assert np.array_equal(getattr(out["fused"], k), getattr(out["split"], k)), k


def test_split_batch_members_identical_alone():
    # a mixed batch group past two loose waves of tiles runs the split shape (batched pair
    # kernel over (solve, tile), solve kernel over (solve, particle block)); each member still
    # ends bit for bit as it does alone
    mk = [lambda: lssph.make_params(lssph.cavity_params(num=128), lanes=4),
          lambda: lssph.make_params(lssph.taylor_green_params(num=128), lanes=4),
          lambda: lssph.make_params(lssph.boussinesq_params(num=96), lanes=4)]
    solo = [_sim(f(), lssph.PRECISION_MIXED, seed=i) for i, f in enumerate(mk)]
    mem = [_sim(f(), lssph.PRECISION_MIXED, seed=i) for i, f in enumerate(mk)]
    with lssph.Batch() as b:
        for m in mem:
            b.add(m)
        b.step(4)
    for s in solo:
        s.step(4)
    for s, m in zip(solo, mem):
        gs, gm = s.download(), m.download()
        for k in _fields(s.params):
            assert np.array_equal(getattr(gs, k), getattr(gm, k)), k
