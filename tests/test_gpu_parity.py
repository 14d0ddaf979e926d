"""Parity of the CUDA engine with the CPU oracle (needs a B200).

Tolerances:
  * lanes = 1 (one thread per particle, reference summation order): results must be
    bit-identical to the oracle (same operation sequence, explicit FMAs only);
  * lanes = 2 / 4 / 8 (warp-shuffle reductions; 0 lets the engine pick 2 or 4): single-stage
    results within a relative 1e-12 of the field scale; whole runs within relative L2
    1e-10 (the stated bound).
Neighbour sets are compared exactly as sorted index sets.
"""
import numpy as np
import pytest

import lssph
import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "u", "v", "rho", "pre")


def _perturbed(p, amp=0.1, seed=0):
    st, ni = lssph.setup_particles(p)
    rng = np.random.default_rng(seed)
    if p.target_problem != 1:
        st.x[:ni] += amp * p.dx * (2 * rng.random(ni) - 1)
        st.y[:ni] += amp * p.dx * (2 * rng.random(ni) - 1)
    return st, ni


def _pair(p, lanes, amp=0.1, seed=0):
    q = lssph.make_params(p, lanes=lanes)
    st, ni = _perturbed(q, amp, seed)
    sim = lssph.Simulation(q, st, ni)
    sim.ghost()
    orc = O.Oracle(q, st, ni, ghost=True)
    return sim, orc


def _rel_l2(a, b):
    d = np.linalg.norm(a - b)
    s = np.linalg.norm(b)
    return d / s if s > 0 else d


CASES = {
    "diffusion": lambda: lssph.diffusion_params(num=50, seed=1),
    "taylor_green": lambda: lssph.taylor_green_params(num=64),
    "cavity": lambda: lssph.cavity_params(num=48),
    "boussinesq": lambda: lssph.boussinesq_params(num=48, ra=1e5),
}


@pytest.mark.parametrize("case", list(CASES))
def test_neighbour_sets_are_bit_exact(case):
    p = CASES[case]()
    sim, orc = _pair(p, lanes=4, amp=0.3, seed=2)
    for which in (0, 1):
        off_g, idx_g = sim.neighbors(which)
        off_o, idx_o = orc.neighbors(which)
        assert np.array_equal(off_g, off_o), which
        assert np.array_equal(idx_g, idx_o), which


@pytest.mark.parametrize("case", list(CASES))
def test_ghost_values(case):
    p = CASES[case]()
    for lanes in (1, 4):
        sim, orc = _pair(p, lanes=lanes, amp=0.2, seed=3)
        g = sim.download()
        o = orc.get()
        vg, vo = sim.virtual_markers(), orc.vm()
        ni = sim.num_int
        for k in ("u", "v", "pre") + (("tem",) if p.target_problem == 4 else ()):
            if lanes == 1:
                assert np.array_equal(g.__dict__[k][ni:], o[k][ni:]), (k, lanes)
                assert np.array_equal(vg[k], vo[k]), (k, lanes)
            else:
                scale = max(np.abs(o[k][ni:]).max(), 1e-30)
                assert np.abs(g.__dict__[k][ni:] - o[k][ni:]).max() <= 1e-12 * scale, (k, lanes)


@pytest.mark.parametrize("case", list(CASES))
def test_single_rhs(case):
    p = CASES[case]()
    for lanes in (1, 4):
        sim, orc = _pair(p, lanes=lanes, amp=0.2, seed=4)
        sim.calculate_rhs()
        orc.calculate_rhs()
        rg, ro = sim.rhs(), orc.rhs()
        keys = ("u",) if p.target_problem == 1 else ("u", "v", "rho") + (("tem",) if p.target_problem == 4 else ())
        for k in keys:
            if lanes == 1:
                assert np.array_equal(rg[k], ro[k]), (k, lanes)
            else:
                scale = max(np.abs(ro[k]).max(), 1e-30)
                assert np.abs(rg[k] - ro[k]).max() <= 1e-12 * scale, (k, lanes)


@pytest.mark.parametrize("case,nsteps", [("diffusion", 50), ("taylor_green", 10), ("cavity", 10),
                                         ("boussinesq", 10)])
def test_steps_bit_exact_with_one_lane(case, nsteps):
    p = CASES[case]()
    sim, orc = _pair(p, lanes=1, amp=0.1, seed=5)
    sim.step(nsteps)
    orc.run(nsteps)
    g, o = sim.download(), orc.get()
    for k in FIELDS + (("tem",) if p.target_problem == 4 else ()):
        assert np.array_equal(getattr(g, k), o[k]), k


def test_operators_equal_fused_step():
    # rk4 + pst called one by one == the graph-replayed step (main.f90:124-134)
    p = lssph.taylor_green_params(num=48)
    a, _ = _pair(p, lanes=4, seed=6)
    b, _ = _pair(p, lanes=4, seed=6)
    for _ in range(3):
        a.rk4()
        a.pst()
    b.step(3)
    ga, gb = a.download(), b.download()
    for k in FIELDS:
        assert np.array_equal(getattr(ga, k), getattr(gb, k)), k


def test_diffusion_1000_steps_rel_l2():
    # configuration 1 (50^2, RK2, jitter 0.05 dx, dt = 0.1 dx^2, 1000 steps): rel L2 <= 1e-10
    p = lssph.diffusion_params(num=50, pos_pert=0.05, coe_dif=0.1, seed=0)
    sim, orc = _pair(p, lanes=4)
    sim.step(1000)
    orc.run(1000)
    g, o = sim.download(), orc.get()
    assert _rel_l2(g.u, o["u"]) <= 1e-10


def test_taylor_green_128_rel_l2():
    # configuration 2 shape (128^2, RK4 + PST, CFL 0.1), 100 steps
    p = lssph.taylor_green_params(num=128)
    sim, orc = _pair(p, lanes=4, amp=0.0)
    sim.step(100)
    orc.run(100)
    g, o = sim.download(), orc.get()
    for k in ("x", "y", "u", "v", "rho"):
        ref = o[k] - (o[k].mean() if k in ("x", "y") else 0.0)
        assert _rel_l2(getattr(g, k), o[k]) <= 1e-10 * max(1.0, np.linalg.norm(o[k]) / max(np.linalg.norm(ref), 1e-300)), k


@pytest.mark.parametrize("case", ["cavity", "boussinesq"])
def test_wall_problems_rel_l2(case):
    p = CASES[case]()
    sim, orc = _pair(p, lanes=4, amp=0.0)
    sim.step(100)
    orc.run(100)
    g, o = sim.download(), orc.get()
    for k in ("u", "v", "pre") + (("tem",) if p.target_problem == 4 else ()):
        assert _rel_l2(getattr(g, k), o[k]) <= 1e-10, k


LANE_CASES = {
    "taylor_green": lambda **kw: lssph.taylor_green_params(num=48, **kw),
    "taylor_green_periodic": lambda **kw: lssph.taylor_green_params(num=48, PERIODIC=1, **kw),
    "cavity": lambda **kw: lssph.cavity_params(num=40, **kw),
    "boussinesq": lambda **kw: lssph.boussinesq_params(num=40, ra=1e5, **kw),
}


@pytest.mark.parametrize("lanes", [2, 8])
@pytest.mark.parametrize("case", list(LANE_CASES))
def test_other_lane_counts_rel_l2(case, lanes):
    # 2 and 8 lanes per particle: the same sums split over another number of lanes, so the
    # same bound as 4 lanes (relative L2 1e-10 over a run)
    p = LANE_CASES[case]()
    sim, orc = _pair(p, lanes=lanes, amp=0.1, seed=7)
    sim.step(60)
    orc.run(60)
    g, o = sim.download(), orc.get()
    assert sim.tuning()["lanes"] == lanes
    for k in ("u", "v", "pre") + (("tem",) if p.target_problem == 4 else ()):
        assert _rel_l2(getattr(g, k), o[k]) <= 1e-10, k


@pytest.mark.parametrize("case", ["taylor_green_periodic_128", "taylor_green_periodic_96", "cavity_64",
                                  "taylor_green_periodic_128_mixed"])
def test_automatic_lanes_equal_the_picked_count(case):
    # lanes = 0: the engine measures 2 and 4 lanes (FP64 q = 5 LS) and keeps the faster; the
    # run is then bit for bit the run with that count given explicitly.  The closed box
    # (ghost launches beside the interior tiles) keeps 4.
    mk = {"taylor_green_periodic_128": lambda **kw: lssph.taylor_green_params(num=128, PERIODIC=1, **kw),
          "taylor_green_periodic_96": lambda **kw: lssph.taylor_green_params(num=96, PERIODIC=1, **kw),
          "cavity_64": lambda **kw: lssph.cavity_params(num=64, **kw),
          "taylor_green_periodic_128_mixed": lambda **kw: lssph.make_params(
              lssph.taylor_green_params(num=128, PERIODIC=1, **kw), precision=lssph.PRECISION_MIXED)}[case]
    auto = lssph.Simulation.new(mk(lanes=0))
    picked = auto.tuning()["lanes"]
    assert picked in (2, 4)
    if auto.tuning()["ghost_overlap"]:
        assert picked == 4
    fixed = lssph.Simulation.new(mk(lanes=picked))
    auto.step(20)
    fixed.step(20)
    ga, gf = auto.download(), fixed.download()
    for k in FIELDS:
        assert np.array_equal(getattr(ga, k), getattr(gf, k)), k
    auto.close()
    fixed.close()


def test_steady_state_detection_matches_oracle():
    # problem 1 stops at max|u_n - u_{n-1}| < THRESHOLD (check_steady_state_mod.f90:39-65)
    p = lssph.diffusion_params(num=20, seed=2, THRESHOLD=2.0e-6)
    sim, orc = _pair(p, lanes=1)
    s_gpu = sim.step(5000)
    s_orc = orc.run(5000)
    assert s_gpu == s_orc and s_gpu > 0
    assert np.array_equal(sim.download().u, orc.get()["u"])
    assert sim.step(10) == 0   # halted at the steady state, like the reference's exit


def test_gpu_error_reports_nonfinite():
    p = lssph.taylor_green_params(num=32)
    st, ni = lssph.setup_particles(p)
    st.u[10] = np.nan
    sim = lssph.Simulation(p, st, ni)
    sim.ghost()
    with pytest.raises(lssph.LssphError) as e:
        sim.step(1)
    assert e.value.status == lssph._abi.E_NONFINITE


def test_snapshot_files(tmp_path):
    p = lssph.taylor_green_params(num=32, SAVE_NAME="tg32")
    sim = lssph.Simulation.new(p)
    sim.write_param(str(tmp_path))
    sim.write_data(str(tmp_path), 0)
    sim.step(3)
    sim.write_data(str(tmp_path), 3)
    base = tmp_path / "tg32"
    assert (base / "config" / "parameters.csv").exists()
    back = lssph.read_data(str(base / "data" / "3.dat"), p)
    g = sim.download()
    for k in FIELDS:
        assert np.array_equal(getattr(back, k), getattr(g, k)), k
    cell = np.fromfile(base / "data" / "cell_idx.dat", dtype="<i4")
    orc = O.Oracle(p)
    assert np.array_equal(cell, orc.cells()[0])
    vm = np.fromfile(base / "data" / "VM.dat", dtype="<i4", count=sim.num_ext)
    assert np.array_equal(vm, orc.vm()["ptype"])
    # restart continues exactly (restart_mod.f90:22-53)
    r = lssph.Simulation.restart(p, str(base / "data" / "3.dat"))
    r.step(2)
    sim.step(2)
    ga, gb = r.download(), sim.download()
    for k in FIELDS:
        assert np.allclose(getattr(ga, k), getattr(gb, k), rtol=1e-12, atol=1e-14), k


@pytest.mark.parametrize("case", ["taylor_green", "boussinesq"])
def test_register_budgets_are_bit_identical(case, monkeypatch):
    # the autotuner's two kernel variants differ only in register allocation
    p = CASES[case]()
    out = {}
    for budget in ("loose", "tight", "five"):
        monkeypatch.setenv("LSSPH_REGISTER_BUDGET", budget)
        st, ni = _perturbed(p, 0.1, 4)
        sim = lssph.Simulation(p, st, ni)
        assert sim.tuning()["register_budget"] == budget
        sim.ghost()
        sim.step(4)
        out[budget] = sim.download()
    for k in FIELDS:
        assert np.array_equal(getattr(out["loose"], k), getattr(out["tight"], k)), k
        assert np.array_equal(getattr(out["loose"], k), getattr(out["five"], k)), k
    monkeypatch.delenv("LSSPH_REGISTER_BUDGET")
    t = lssph.Simulation(p, *_perturbed(p, 0.1, 4)).tuning()
    assert t["rhs_us_loose"] > 0 and t["rhs_us_tight"] > 0
    if t["ghost_overlap"] and t["shape"] == "fused":   # the interior tiles share the SMs with the ghost launch
        assert t["register_budget"] == "tight"


def test_overlapped_step_equals_serial_step(monkeypatch):
    # ghost launches beside the next stage's interior tiles change no result
    for case in ("taylor_green", "boussinesq", "diffusion"):
        # lanes fixed: the automatic count is measured on each schedule and may differ
        p = lssph.make_params(CASES[case](), NUM_X=96, NUM_Y=96, lanes=4)
        out = {}
        for ov in ("0", "1"):
            monkeypatch.setenv("LSSPH_OVERLAP", ov)
            st, ni = _perturbed(p, 0.1, 7)
            sim = lssph.Simulation(p, st, ni)
            sim.ghost()
            assert sim.tuning()["ghost_overlap"] == (ov == "1"), case
            sim.step(6)
            out[ov] = sim.download()
        for k in FIELDS + (("tem",) if p.target_problem == 4 else ()):
            assert np.array_equal(getattr(out["0"], k), getattr(out["1"], k)), (case, k)


# ---- the FP64 split shape --------------------------------------------------------------
# The split shape runs the fused kernels' pair phase in a pair kernel (sums to device
# memory) and their solve and update in a kernel with one thread per particle; per particle
# the arithmetic is the fused kernels', so both shapes give the same bits.
@pytest.mark.parametrize("lanes", [2, 4])
@pytest.mark.parametrize("case", list(CASES))
def test_fp64_split_and_fused_shapes_give_identical_bits(case, lanes, monkeypatch):
    p = lssph.make_params(CASES[case](), lanes=lanes)
    out = {}
    for shape in ("fused", "split"):
        monkeypatch.setenv("LSSPH_KERNEL_SHAPE", shape)
        st, ni = _perturbed(p, 0.1, 5)
        sim = lssph.Simulation(p, st, ni)
        sim.ghost()
        sim.step(6)
        assert sim.tuning()["shape"] == shape
        out[shape] = sim.download()
        sim.close()
    for k in FIELDS + (("tem",) if p.target_problem == 4 else ()):
        assert np.array_equal(getattr(out["fused"], k), getattr(out["split"], k)), (case, k)


@pytest.mark.parametrize("budget", ["loose", "tight", "five", "six", "eight"])
def test_fp64_split_budgets_match_the_oracle(budget, monkeypatch):
    # every register budget of the FP64 pair kernel (six and eight spill), on the periodic
    # Taylor-Green square, against the oracle
    monkeypatch.setenv("LSSPH_KERNEL_SHAPE", "split")
    monkeypatch.setenv("LSSPH_REGISTER_BUDGET", budget)
    p = lssph.taylor_green_params(num=64, re=100.0, coe_cfl=0.1, tg=2, lanes=2, PERIODIC=1)
    st, ni = lssph.setup_particles(p)
    sim = lssph.Simulation(p, st, ni)
    orc = O.Oracle(p, st, ni, ghost=False)
    sim.step(40)
    orc.run(40)
    t = sim.tuning()
    assert t["shape"] == "split" and t["register_budget"] == budget
    g, o = sim.download(), orc.get()
    for k in ("x", "y", "u", "v", "pre"):
        assert _rel_l2(getattr(g, k), o[k]) <= 1e-10, k
    sim.close()


def test_fp64_split_batch_members_identical_alone(monkeypatch):
    # members that picked the split shape alone make their batch group run it (batched FP64
    # pair kernel over (solve, tile), solve kernel over (solve, particle block)); each member
    # still ends bit for bit as it does alone
    monkeypatch.setenv("LSSPH_KERNEL_SHAPE", "split")
    mk = [lambda: lssph.make_params(lssph.cavity_params(num=64), lanes=4),
          lambda: lssph.make_params(lssph.taylor_green_params(num=64), lanes=4),
          lambda: lssph.make_params(lssph.boussinesq_params(num=48), lanes=4)]
    solo, mem = [], []
    for i, f in enumerate(mk):
        for group in (solo, mem):
            p = f()
            st, ni = _perturbed(p, 0.1, 10 + i)
            sim = lssph.Simulation(p, st, ni)
            sim.ghost()
            sim.step(1)   # the first solo launch measures (here: fixes) the shape
            assert sim.tuning()["shape"] == "split"
            group.append(sim)
    with lssph.Batch() as b:
        for m in mem:
            b.add(m)
        b.step(4)
    for s in solo:
        s.step(4)
    for s, m in zip(solo, mem):
        gs, gm = s.download(), m.download()
        for k in FIELDS + (("tem",) if s.params.target_problem == 4 else ()):
            assert np.array_equal(getattr(gs, k), getattr(gm, k)), k
        s.close()
        m.close()


# ---- the autotuner's measurement leaves no trace -------------------------------------------
@pytest.mark.parametrize("case", ["periodic", "cavity"])
def test_measurement_leaves_no_trace(case, monkeypatch):
    # the first launch times whole steps of every option on the solve's own state and puts
    # the state back (step budget and step count included); a budget of 3 set before that
    # launch still stops the solve after exactly 3 steps, at the state that a run with the
    # picked configuration fixed (no measurement) reaches
    monkeypatch.delenv("LSSPH_KERNEL_SHAPE", raising=False)
    monkeypatch.delenv("LSSPH_REGISTER_BUDGET", raising=False)
    base = (lssph.taylor_green_params(num=48, PERIODIC=1, coe_cfl=0.1) if case == "periodic"
            else lssph.cavity_params(num=48))
    st, ni = _perturbed(base, 0.1, 21)
    a = lssph.Simulation(base, st, ni)
    a.ghost()
    a.set_step_budget(3)
    a.step(10)
    assert a.progress() == (3, "budget")
    t = a.tuning()
    monkeypatch.setenv("LSSPH_KERNEL_SHAPE", t["shape"])
    monkeypatch.setenv("LSSPH_REGISTER_BUDGET", t["register_budget"])
    b = lssph.Simulation(lssph.make_params(base, lanes=t["lanes"]), st, ni)
    b.ghost()
    b.step(3)
    ga, gb = a.download(), b.download()
    for k in FIELDS:
        assert np.array_equal(getattr(ga, k), getattr(gb, k)), (k, t)
    a.close()
    b.close()
