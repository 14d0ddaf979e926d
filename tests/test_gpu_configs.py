"""Parity at the benchmarked configurations, at their own sizes and horizons (needs a B200).

  * configuration 2 as the bench times it: periodic Taylor-Green, Re = 100, 128^2, RK4 +
    PST, CFL 0.1, with the engine's automatic lane count, each kernel shape and each register
    budget, against the oracle after 120 steps (rel L2 <= 1e-10);
  * configuration 1 as written (periodic 50^2 diffusion, jitter +-0.05 dx, dt = 0.1 dx^2,
    RK2, 1000 steps) and configuration 2 to t = 1 (12,800 steps): with one lane per particle
    (the reference's summation order) every field is bit-identical to the oracle's at the
    end; with the automatic lane count the error against the analytic decay equals the
    oracle's within the bound stated at each test;
  * the sensitivity horizon: a one-ulp change of the positions grows in the oracle itself
    as fast as the GPU's 2-lane vs 4-lane difference, so beyond it two correct FP64 runs
    differ at the field level and only statistics such as the analytic error compare.

The oracle runs on all host cores; the 12,800-step run takes a few minutes.
"""
import os

import numpy as np
import pytest

import lssph
import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "u", "v", "rho", "pre")
STEPS_T1 = 12800   # t = 1 at dt = 0.1 dx / c = 7.8125e-5 (128^2, c = 10)


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def tg_params(lanes, num=128):
    return lssph.taylor_green_params(num=num, re=100.0, coe_cfl=0.1, tg=2, lanes=lanes, PERIODIC=1)


def tg_velocity_error(st, p, nsteps):
    """Velocity rel. L2 against u = sin 2pi x cos 2pi y exp(-8 pi^2 nu t) (and v), the decay of
    analysis/benchmarks/taylor_green.py:35 for TG_A = TG_B = 2."""
    t = nsteps * p.dt
    dec = np.exp(-8.0 * np.pi ** 2 * p.kinematic_vis * t)
    x, y = np.asarray(st["x"]), np.asarray(st["y"])
    ue = np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) * dec
    ve = -np.cos(2 * np.pi * x) * np.sin(2 * np.pi * y) * dec
    u, v = np.asarray(st["u"]), np.asarray(st["v"])
    return float(np.sqrt((np.sum((u - ue) ** 2) + np.sum((v - ve) ** 2)) / (np.sum(ue ** 2) + np.sum(ve ** 2))))


def _as_dict(st):
    return {k: getattr(st, k) for k in FIELDS}


@pytest.fixture(scope="module", autouse=True)
def _all_cores():
    O.set_threads(os.cpu_count() or 1)


HEADLINE_KERNELS = ([(0, None, None)] + [(g, b, "fused") for g in (2, 4) for b in ("loose", "tight", "five")] +
                    [(g, b, "split") for g in (2, 4) for b in ("loose", "tight", "five", "six")])


@pytest.mark.parametrize("lanes,budget,shape", HEADLINE_KERNELS)
def test_headline_workload_matches_the_oracle(lanes, budget, shape, monkeypatch):
    # the kernels the bench may time: lanes = 0 lets the engine pick 2 or 4, the kernel shape
    # and the register budget by measurement (what the bench runs); the explicit cases cover
    # every pick
    for var, val in (("LSSPH_REGISTER_BUDGET", budget), ("LSSPH_KERNEL_SHAPE", shape)):
        if val:
            monkeypatch.setenv(var, val)
        else:
            monkeypatch.delenv(var, raising=False)
    p = tg_params(lanes=lanes)
    st, ni = lssph.setup_particles(p)
    sim = lssph.Simulation(p, st, ni)
    orc = O.Oracle(p, st, ni, ghost=False)
    sim.step(120)
    orc.run(120)
    tune = sim.tuning()
    if budget:
        assert tune["register_budget"] == budget and tune["lanes"] == lanes and tune["shape"] == shape
    g, o = sim.download(), orc.get()
    for k in ("x", "y", "u", "v", "pre"):
        assert _rel_l2(getattr(g, k), o[k]) <= 1e-10, (k, tune)
    sim.close()


# ---- configuration 1 as written --------------------------------------------------------
def diffusion_cfg1(lanes, seed=11):
    return lssph.diffusion_params(num=50, pos_pert=0.05, coe_dif=0.1, seed=seed, lanes=lanes, PERIODIC=1)


def diffusion_error(st, p, nsteps):
    """Rel. L2 of u against sin 2pi x sin 2pi y exp(-8 pi^2 t) (alpha = 1)."""
    x, y, u = (np.asarray(st[k]) for k in ("x", "y", "u"))
    ex = np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y) * np.exp(-8 * np.pi ** 2 * nsteps * p.dt)
    return _rel_l2(u, ex)


@pytest.fixture(scope="module")
def cfg1_oracle():
    p = diffusion_cfg1(lanes=1)
    assert abs(p.dt - 0.1 * p.dx ** 2) <= 1e-15 * p.dt and p.rk == 2
    st, ni = lssph.setup_particles(p)
    orc = O.Oracle(p, st, ni, ghost=False)
    orc.run(1000)
    return p, st, ni, orc.get()


def test_configuration_1_bit_identical_after_1000_steps(cfg1_oracle):
    p, st, ni, o = cfg1_oracle
    sim = lssph.Simulation(p, st, ni)
    sim.step(1000)
    g = sim.download()
    for k in FIELDS:
        assert np.array_equal(getattr(g, k), o[k]), k
    sim.close()


def test_configuration_1_analytic_error_equals_the_oracles(cfg1_oracle):
    # positions are fixed in problem 1 and the update is linear in u, so the automatic lane
    # count changes the result only at the rounding level: the two errors against the
    # analytic decay agree to 1e-9 of themselves
    p, st, ni, o = cfg1_oracle
    q = diffusion_cfg1(lanes=0)
    sim = lssph.Simulation(q, st, ni)
    sim.step(1000)
    g = _as_dict(sim.download())
    e_gpu, e_orc = diffusion_error(g, p, 1000), diffusion_error(o, p, 1000)
    assert 0 < e_orc < 0.05   # 1.2e-2 at t = 0.04 on the jittered 50^2 lattice
    assert abs(e_gpu - e_orc) <= 1e-9 * e_orc, (e_gpu, e_orc)
    assert _rel_l2(g["u"], o["u"]) <= 1e-10
    sim.close()


# ---- configuration 2 to t = 1 -----------------------------------------------------------
@pytest.fixture(scope="module")
def cfg2_oracle():
    p = tg_params(lanes=1)
    assert abs(STEPS_T1 * p.dt - 1.0) < 1e-12
    st, ni = lssph.setup_particles(p)
    orc = O.Oracle(p, st, ni, ghost=False)
    orc.run(STEPS_T1)
    return p, st, ni, orc.get()


def test_configuration_2_to_t1_bit_identical_with_one_lane(cfg2_oracle):
    p, st, ni, o = cfg2_oracle
    sim = lssph.Simulation(p, st, ni)
    sim.step(STEPS_T1)
    g = sim.download()
    for k in FIELDS:
        assert np.array_equal(getattr(g, k), o[k]), k
    sim.close()


def test_configuration_2_to_t1_analytic_error_equals_the_oracles(cfg2_oracle):
    # past the sensitivity horizon (below) the automatic lane count and the reference order
    # give different particle arrangements, so only the error against the analytic decay
    # compares: equal within 5 % of itself
    p, st, ni, o = cfg2_oracle
    e_orc = tg_velocity_error(o, p, STEPS_T1)
    sim = lssph.Simulation(tg_params(lanes=0), st, ni)
    sim.step(STEPS_T1)
    g = _as_dict(sim.download())
    e_gpu = tg_velocity_error(g, p, STEPS_T1)
    assert 0 < e_orc < 0.05
    assert abs(e_gpu - e_orc) <= 0.05 * e_orc, (e_gpu, e_orc, sim.tuning())
    sim.close()


# ---- the sensitivity horizon -------------------------------------------------------------
def test_sensitivity_horizon_is_the_algorithms_own():
    # one ulp on every position grows in the oracle as the GPU's 2- vs 4-lane summation
    # order difference does: both stay below 1e-10 for 500 steps and pass 1e-5 by 1000
    p = tg_params(lanes=1)
    st, ni = lssph.setup_particles(p)
    st2 = st.copy()
    st2.x[:] = np.nextafter(st2.x, 2.0)
    a, b = O.Oracle(p, st, ni, ghost=False), O.Oracle(p, st2, ni, ghost=False)
    s2 = lssph.Simulation(tg_params(lanes=2), st, ni)
    s4 = lssph.Simulation(tg_params(lanes=4), st, ni)
    d = {}
    done = 0
    for n in (500, 1000):
        a.run(n - done)
        b.run(n - done)
        s2.step(n - done)
        s4.step(n - done)
        done = n
        oa, ob = a.get(), b.get()
        g2, g4 = s2.download(), s4.download()
        d[n] = (_rel_l2(ob["u"], oa["u"]), _rel_l2(g2.u, g4.u))
    assert d[500][0] < 1e-10 and d[500][1] < 1e-10, d
    assert d[1000][0] > 1e-5 and d[1000][1] > 1e-5, d
    s2.close()
    s4.close()
