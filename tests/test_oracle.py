"""The CPU oracle against the reference's golden vectors and analytic known answers
(no GPU).  These pin the checker before any engine result is compared with it."""
import numpy as np
import pytest
import scipy.linalg

import lssph
import oracle as O


def test_kernel_functions_match_reference_python(golden_dir):
    # kernel_functions_mod.f90:26-81 vs analysis/common/kernel_functions.py
    g = np.load(f"{golden_dir}/kernels.npz")
    h = float(g["h"])
    for kt in range(1, 6):
        mine = np.array([O.kernel_W(kt, r, h) for r in g["r"]])
        ref = g["W"][kt - 1]
        assert np.max(np.abs(mine - ref)) <= 4e-15 * np.max(np.abs(ref)), kt


def test_kernel_derivative_is_consistent():
    # cal_dW (kernel_functions_mod.f90:87-146) is the r-derivative of cal_W
    h = 0.012
    for kt in range(1, 6):
        for r in np.linspace(0.05 * h, 1.95 * h, 17):
            eps = 1e-7 * h
            fd = (O.kernel_W(kt, r + eps, h) - O.kernel_W(kt, r - eps, h)) / (2 * eps)
            assert O.kernel_dW(kt, r, h) == pytest.approx(fd, rel=2e-6, abs=1e-6 * abs(O.kernel_W(kt, 0.0, h)) / h)


@pytest.mark.parametrize("q", [3, 6])
def test_lssph_b_matches_reference_python(golden_dir, q):
    # interpolate_LSSPH_B math vs analysis/common/lssph_b.py:21-143
    b = np.load(f"{golden_dir}/lssph_b.npz")
    p = lssph.make_params(NUM_X=50, NUM_Y=50)   # dx = 0.02, h = 0.024, Wendland C2
    assert p.dx == float(b["dx"])
    out = O.lssph_b(p, q, b["xs"], b["ys"], b["rho"], b["val"], b["xt"], b["yt"])
    np.testing.assert_allclose(out, b[f"q{q}"], rtol=0, atol=1e-13)


# Post-processing LS-B (analysis/common/lssph_b.py:21-143) against the reference's own
# output for every basis size.  The reference forms A^T W A with BLAS, the restatement sums
# neighbour by neighbour, so the two differ by rounding amplified by the conditioning of
# the normal equations: bounds per q, relative to each output column's largest value.
POST_TOL = {3: 1e-12, 6: 1e-10, 10: 1e-9, 15: 5e-9, 21: 5e-9}


def post_params(case):
    tp, sm, kt, h, he = case
    p = lssph.make_params(NUM_X=50, NUM_Y=50)
    p.target_problem, p.sph_model, p.kernel_type = int(tp), int(sm), int(kt)
    p.h, p.h_eff, p.SP_mass = float(h), float(he), 0.02 ** 2
    return p


@pytest.mark.parametrize("i", range(8))
def test_lsb_post_matches_reference_python(golden_dir, i):
    g = np.load(f"{golden_dir}/lssph_b_post.npz")
    p = post_params(g["cases"][i])
    q = {2: 3, 4: 6}[p.target_problem] if p.sph_model <= 3 else \
        {(4, 2): 6, (4, 4): 10, (5, 2): 10, (5, 4): 15, (6, 2): 15, (6, 4): 21}[(p.sph_model, p.target_problem)]
    out = O.lsb_post(p, g["xt"], g["yt"], g["xs"], g["ys"], g["val"], g["rho"])
    ref = g[f"case{i}"]
    assert np.array_equal(np.isnan(out), np.isnan(ref))
    ok = ~np.isnan(ref[:, 0])
    assert ok.sum() >= 30
    err = np.abs(out[ok] - ref[ok]).max(axis=0) / np.abs(ref[ok]).max(axis=0)
    assert (err <= POST_TOL[q]).all(), (q, err)


@pytest.mark.parametrize("n,nrhs", [(3, 3), (3, 4), (5, 4), (5, 5), (6, 4), (9, 3)])
def test_dgesv_restatement_matches_lapack(n, nrhs):
    rng = np.random.default_rng(n * 10 + nrhs)
    for _ in range(20):
        X = rng.standard_normal((n, 2 * n))
        A = X @ np.diag(rng.random(2 * n) + 0.1) @ X.T     # SPD-like moment matrix
        A[0, :] *= 1e-3                                   # force pivoting
        B = rng.standard_normal((n, nrhs))
        mine, info = O.dgesv(A, B)
        lu, piv, ref, inf = scipy.linalg.lapack.dgesv(A, B)
        assert info == 0 and inf == 0
        np.testing.assert_allclose(mine, ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max())


def test_dgesv_reports_singular_pivot():
    A = np.array([[1.0, 2.0, 3.0], [2.0, 4.0, 6.0], [1.0, 0.0, 1.0]])
    _, info = O.dgesv(A, np.ones(3))
    assert info > 0


def _quadratic_fields(x, y):
    u = 0.3 + 1.1 * x - 0.7 * y + 2.0 * x * x - 1.5 * x * y + 0.8 * y * y
    v = -0.2 + 0.4 * x + 0.9 * y - 1.0 * x * x + 0.6 * x * y + 1.2 * y * y
    return u, v


def test_ls_type_a_reproduces_quadratics_exactly():
    # LSSPH_A (q = 5) differentiates any quadratic exactly on any cloud with >= 5
    # neighbours: d/dx, d/dy exact, Laplacian exact.
    p = lssph.make_params(TARGET_PROBLEM=2, NUM_X=24, NUM_Y=24, TG_A=2, TG_B=2, COE_DELTA_SPH=0.0)
    st, ni = lssph.setup_particles(p)
    rng = np.random.default_rng(7)
    st.x[:ni] += 0.1 * p.dx * (2 * rng.random(ni) - 1)
    st.y[:ni] += 0.1 * p.dx * (2 * rng.random(ni) - 1)
    st.u, st.v = _quadratic_fields(st.x, st.y)
    st.rho = np.full_like(st.x, p.rho_ref)
    st.pre = 0.5 * st.x + 0.25 * st.y     # linear pressure: grad = (0.5, 0.25)
    o = O.Oracle(p, st, ni, ghost=False)
    o.calculate_rhs()
    r = o.rhs()
    x, y = st.x[:ni], st.y[:ni]
    lap_u = 2 * 2.0 + 2 * 0.8
    lap_v = 2 * -1.0 + 2 * 1.2
    div = (1.1 + 4.0 * x - 1.5 * y) + (0.9 + 0.6 * x + 2.4 * y)
    # RHS_u = -p_x/rho + (mu/rho) lap u, RHS_rho = -rho div u (LSSPH_A_mod.f90:253-255)
    np.testing.assert_allclose(r["u"], -0.5 + p.vis_ref * lap_u, rtol=0, atol=1e-8)
    np.testing.assert_allclose(r["v"], -0.25 + p.vis_ref * lap_v, rtol=0, atol=1e-8)
    np.testing.assert_allclose(r["rho"], -div, rtol=0, atol=1e-9)


def test_oracle_threads_are_bit_identical():
    p = lssph.taylor_green_params(num=32, end_step=100)
    O.set_threads(1)
    a = O.Oracle(p)
    a.run(3)
    O.set_threads(8)
    b = O.Oracle(p)
    b.run(3)
    ga, gb = a.get(), b.get()
    for k in ("x", "y", "u", "v", "rho", "pre"):
        assert np.array_equal(ga[k], gb[k]), k


def test_oracle_neighbour_sets_match_brute_force():
    p = lssph.diffusion_params(num=20, seed=11, pos_pert=0.2)
    o = O.Oracle(p)
    off, idx = o.neighbors(0)
    g = o.get()
    x, y = g["x"], g["y"]
    h2 = p.h_eff * p.h_eff
    for i in range(0, o.num_int, 7):
        dx = x - x[i]
        dy = y - y[i]
        brute = np.nonzero(dx * dx + dy * dy <= h2)[0]
        brute = brute[brute != i]
        assert np.array_equal(np.sort(brute), idx[off[i]:off[i + 1]])


def test_diffusion_transient_follows_analytic_solution():
    # u_t = lap u + 2 pi^2 phi, u(0) = 0, phi = sin(pi x) cos(pi y) (LSSPH_A_mod.f90:247).
    # With Dirichlet u = 0 on the left/right walls and Neumann du/dy = 0 on the top/bottom
    # walls (extrapolate_diff_test_mod.f90:40-103) phi meets every wall condition, so
    # u = phi (1 - exp(-2 pi^2 t)) exactly.
    p = lssph.diffusion_params(num=30, pos_pert=0.05, seed=1, bc_tb=1, bc_lr=2)
    o = O.Oracle(p)
    nsteps = 400
    o.run(nsteps)
    g = o.get()
    ni = o.num_int
    x = g["x"][:ni] - p.WL_thick
    y = g["y"][:ni] - p.WL_thick
    t = nsteps * p.dt
    exact = np.sin(np.pi * x) * np.cos(np.pi * y) * (1 - np.exp(-2 * np.pi ** 2 * t))
    err = np.sqrt(np.mean((g["u"][:ni] - exact) ** 2))
    assert err < 5e-3 * np.max(np.abs(exact))   # LS Laplacian is 1st-order accurate at 30^2


def test_taylor_green_decays_at_the_analytic_rate():
    # kinetic energy ~ exp(-2 sigma t), sigma = nu ((a pi)^2 + (b pi)^2) (taylor_green.py:35)
    p = lssph.taylor_green_params(num=48, re=100.0, tg=2, coe_cfl=0.1)
    o = O.Oracle(p)
    g0 = o.get()
    ni = o.num_int
    e0 = np.sum(g0["u"][:ni] ** 2 + g0["v"][:ni] ** 2)
    n = 200
    o.run(n)
    g = o.get()
    e = np.sum(g["u"][:ni] ** 2 + g["v"][:ni] ** 2)
    sigma = p.kinematic_vis * 2 * (2 * np.pi) ** 2
    expect = np.exp(-2 * sigma * n * p.dt)
    assert e / e0 == pytest.approx(expect, rel=2e-2)


# Periodic-domain extension (no counterpart in the reference, so not reference-pinned):
# pinned to the analytic solutions instead.
def test_periodic_diffusion_decays_at_the_analytic_rate():
    # u = sin(2 pi x) sin(2 pi y) exp(-8 pi^2 t) with nu = 1, on the jittered lattice
    errs = []
    for num in (32, 64):
        p = lssph.diffusion_params(num=num, seed=3, PERIODIC=1)
        orc = O.Oracle(p)
        n = 100
        orc.run(n)
        o, ni = orc.get(), orc.num_int
        assert orc.num_total == ni == num * num          # no ghost particles
        ex = np.sin(2 * np.pi * o["x"][:ni]) * np.sin(2 * np.pi * o["y"][:ni]) * np.exp(-8 * np.pi ** 2 * n * p.dt)
        errs.append(np.linalg.norm(o["u"][:ni] - ex) / np.linalg.norm(ex))
    assert errs[1] < 5e-3 and errs[1] < errs[0] / 3      # converges with resolution


def test_periodic_taylor_green_decays_at_the_analytic_rate():
    p = lssph.taylor_green_params(num=64, PERIODIC=1)
    orc = O.Oracle(p)
    n = 200
    orc.run(n)
    o = orc.get()
    amp = np.sqrt(np.mean(o["u"] ** 2 + o["v"] ** 2) / 0.5)
    exact = np.exp(-8 * np.pi ** 2 * p.kinematic_vis * n * p.dt)
    assert abs(amp - exact) < 2e-3
    assert (o["x"] > 0).all() and (o["x"] <= p.len_x).all() and (o["y"] > 0).all() and (o["y"] <= p.len_y).all()


def test_periodic_rejects_wall_problems():
    with pytest.raises(lssph.LssphError):
        lssph.cavity_params(num=32, PERIODIC=1)


def _poly_case(sm, deg, kw):
    # a random polynomial of degree `deg` on a jittered problem-1 lattice, and its Laplacian
    p = lssph.diffusion_params(num=30, pos_pert=0.2, seed=7, SPH_MODEL=sm, **kw)
    st, ni = lssph.setup_particles(p)
    X, Y = st.x - p.WL_thick, st.y - p.WL_thick
    rng = np.random.default_rng(sm)
    coef = {(i, j): rng.normal() for i in range(deg + 1) for j in range(deg + 1 - i)}
    st.u[:] = sum(c * X ** i * Y ** j for (i, j), c in coef.items())
    lap = sum(c * (i * (i - 1) * X ** max(i - 2, 0) * Y ** j + j * (j - 1) * X ** i * Y ** max(j - 2, 0))
              for (i, j), c in coef.items())
    x, y = st.x[:ni], st.y[:ni]
    src = 2 * np.pi ** 2 * np.sin(np.pi * (x - p.WL_thick)) * np.cos(np.pi * (y - p.WL_thick))
    return p, st, ni, lap[:ni], src


POLY_CASES = [(3, 2, {}), (4, 3, {}), (5, 4, {}), (6, 5, {"KERNEL_TYPE": 2})]


@pytest.mark.parametrize("sm,deg,kw", POLY_CASES)
def test_ls_type_a_reproduces_polynomials_of_its_order(sm, deg, kw):
    # order-k LS (SPH_MODEL 3..6) differentiates degree-k polynomials exactly on any cloud
    # with enough neighbours: problem 1's RHS minus its source is the exact Laplacian
    p, st, ni, lap, src = _poly_case(sm, deg, kw)
    o = O.Oracle(p, st, ni, ghost=False)
    o.calculate_rhs()
    err = np.abs((o.rhs()["u"] - src) - lap).max() / np.abs(lap).max()
    assert err < 1e-10, err


def test_ls_type_b_interpolates_linear_fields_exactly():
    # LS type B (q = 3, interpolate_LSSPH_B_mod.f90) reproduces a linear field exactly at
    # every virtual marker (fluid-only neighbours)
    p = lssph.cavity_params(num=32)
    st, ni = lssph.setup_particles(p)
    rng = np.random.default_rng(3)
    st.x[:ni] += 0.15 * p.dx * (2 * rng.random(ni) - 1)
    st.y[:ni] += 0.15 * p.dx * (2 * rng.random(ni) - 1)
    st.u[:] = 0.3 + 1.7 * st.x - 0.4 * st.y
    st.v[:] = -0.2 + 0.5 * st.x + 2.1 * st.y
    st.pre[:] = 1.0 - 3.0 * st.x + 0.25 * st.y
    o = O.Oracle(p, st, ni, ghost=True)
    vm = o.vm()
    np.testing.assert_allclose(vm["u"], 0.3 + 1.7 * vm["x"] - 0.4 * vm["y"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(vm["v"], -0.2 + 0.5 * vm["x"] + 2.1 * vm["y"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(vm["pre"], 1.0 - 3.0 * vm["x"] + 0.25 * vm["y"], rtol=0, atol=1e-11)


def test_oracle_amplifies_one_ulp_in_the_positions():
    # the sensitivity horizon of the reference algorithm itself: periodic Taylor-Green
    # Re = 100, 64^2, RK4 + PST; one ulp added to every position stays at the rounding level
    # for 200 steps and has grown to the percent level of the velocity by 1000.  So two
    # correct FP64 runs that differ only in rounding (summation order, compiler, FMA
    # placement) agree field by field only before that horizon.
    p = lssph.taylor_green_params(num=64, re=100.0, coe_cfl=0.1, tg=2, lanes=1, PERIODIC=1)
    st, ni = lssph.setup_particles(p)
    st2 = st.copy()
    st2.x[:] = np.nextafter(st2.x, 2.0)
    a, b = O.Oracle(p, st, ni, ghost=False), O.Oracle(p, st2, ni, ghost=False)
    rel = {}
    done = 0
    for n in (200, 1000):
        a.run(n - done)
        b.run(n - done)
        done = n
        ua, ub = a.get()["u"], b.get()["u"]
        rel[n] = np.linalg.norm(ub - ua) / np.linalg.norm(ua)
    assert 0 < rel[200] < 1e-12, rel
    assert rel[1000] > 1e-4, rel
