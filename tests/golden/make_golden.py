"""Generate the golden vectors of tests/golden/ from the reference's own Python code.

    python tests/golden/make_golden.py REFERENCE_ROOT
    LSSPH_REFERENCE_ROOT=... python tests/golden/make_golden.py

Needs the LS-SPH-Benchmarks checkout (the argument, else $LSSPH_REFERENCE_ROOT) for
analysis/common/kernel_functions.py and analysis/common/lssph_b.py, plus numpy/scipy.
The fixtures it writes are committed; the tests read only the .npz files.

  kernels.npz   W(r, h) of the five kernels (KERNEL_TYPE 1..5) on a radius grid,
                from kernel_functions.{cubic_spline,quintic_spline,wendland_C2,
                wendland_C4,wendland_C6}_W
  lssph_b.npz   LS type-B (q = 3 and q = 6) interpolation of smooth fields at target
                points over a seeded jittered particle cloud, from lssph_b.main
                (analysis/common/lssph_b.py:21-143), the interpolation the reference
                uses for its virtual markers (interpolate_LSSPH_B_mod.f90)
  lssph_b_post.npz  the full post-processing output of lssph_b.main (value, d/dx, d/dy)
                for every basis size it supports (q = 3, 6, 10, 15, 21: SPH_MODEL x
                TARGET_PROBLEM), several kernels, over a jittered cloud, with targets
                inside, on the edge of and outside the cloud
"""
import os
import sys
from types import SimpleNamespace

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root: str) -> None:
    sys.path.insert(0, ref_root)
    from analysis.common import kernel_functions as kf  # reference code
    from analysis.common import lssph_b  # reference code

    # ---- kernels ------------------------------------------------------------------------
    h = 0.012
    r = np.linspace(0.0, 3.2 * h, 257)
    funcs = [kf.cubic_spline_W, kf.quintic_spline_W, kf.wendland_C2_W, kf.wendland_C4_W, kf.wendland_C6_W]
    W = np.stack([f(r, h) for f in funcs])
    np.savez(os.path.join(HERE, "kernels.npz"), r=r, h=np.array(h), W=W)

    # ---- LS type B ----------------------------------------------------------------------
    rng = np.random.default_rng(20260312)
    dx = 0.02
    n = 24
    gx, gy = np.meshgrid((np.arange(n) + 0.5) * dx, (np.arange(n) + 0.5) * dx)
    xs = gx.ravel() + 0.1 * dx * (2 * rng.random(n * n) - 1)
    ys = gy.ravel() + 0.1 * dx * (2 * rng.random(n * n) - 1)
    rho = 1.0 + 0.01 * np.sin(3.0 * xs) * np.cos(2.0 * ys)
    val = np.sin(2.0 * np.pi * xs) * np.cos(np.pi * ys) + 0.3 * xs * ys
    xt = 0.12 + 0.24 * rng.random(40)
    yt = 0.12 + 0.24 * rng.random(40)
    out = {}
    for target, q in ((2, 3), (4, 6)):
        param = SimpleNamespace(h_eff=2.4 * dx, h=1.2 * dx, target_problem=target, kernel_type=3, sph_model=3,
                                SP_mass=1.0 * dx * dx)
        res = lssph_b.main(param, xt, yt, xs, ys, val, rho)
        out[f"q{q}"] = res[:, 0]
    np.savez(os.path.join(HERE, "lssph_b.npz"), xs=xs, ys=ys, rho=rho, val=val, xt=xt, yt=yt, dx=np.array(dx),
             q3=out["q3"], q6=out["q6"])
    # ---- post-processing LS type B, every basis size -------------------------------------
    rng = np.random.default_rng(20261204)
    n = 20
    gx, gy = np.meshgrid((np.arange(n) + 0.5) * dx, (np.arange(n) + 0.5) * dx)
    xs = gx.ravel() + 0.2 * dx * (2 * rng.random(n * n) - 1)
    ys = gy.ravel() + 0.2 * dx * (2 * rng.random(n * n) - 1)
    rho = 1.0 + 0.02 * np.sin(3.0 * xs) * np.cos(2.0 * ys)
    val = np.sin(2.0 * np.pi * xs) * np.cos(np.pi * ys) + 0.3 * xs * ys
    L = n * dx
    xt = np.concatenate([0.1 * L + 0.8 * L * rng.random(24), [0.0, L, 0.5 * L, -0.2 * L, 0.5 * L],
                         np.linspace(0.0, L, 8)])
    yt = np.concatenate([0.1 * L + 0.8 * L * rng.random(24), [0.5 * L, 0.5 * L, 0.0, 0.5 * L, 1.3 * L],
                         np.full(8, 0.5 * L)])
    cases = []
    # (target_problem, sph_model, kernel_type, h / dx, h_eff / h)
    for tp, sm, kt, ch, he in ((2, 3, 3, 1.2, 2.0), (4, 3, 3, 1.2, 2.0), (2, 4, 1, 1.5, 2.0), (4, 4, 4, 1.5, 2.0),
                               (2, 5, 5, 2.0, 2.0), (4, 5, 2, 1.2, 3.0), (2, 6, 2, 1.4, 3.0), (4, 6, 3, 2.2, 2.0)):
        h = ch * dx
        param = SimpleNamespace(h_eff=he * h, h=h, target_problem=tp, kernel_type=kt, sph_model=sm,
                                SP_mass=1.0 * dx * dx)
        cases.append([tp, sm, kt, h, he * h])
        out[f"case{len(cases) - 1}"] = lssph_b.main(param, xt, yt, xs, ys, val, rho)
    np.savez(os.path.join(HERE, "lssph_b_post.npz"), xs=xs, ys=ys, rho=rho, val=val, xt=xt, yt=yt,
             dx=np.array(dx), cases=np.array(cases), **{k: v for k, v in out.items() if k.startswith("case")})
    print("wrote", os.path.join(HERE, "kernels.npz"), os.path.join(HERE, "lssph_b.npz"),
          os.path.join(HERE, "lssph_b_post.npz"))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LSSPH_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py REFERENCE_ROOT (or set LSSPH_REFERENCE_ROOT)")
    main(root)
