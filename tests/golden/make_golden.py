"""Generate the golden vectors of tests/golden/ from the reference's own Python code.

    python tests/golden/make_golden.py [REFERENCE_ROOT]

Needs the LS-SPH-Benchmarks checkout (default /root/reference) for
analysis/common/kernel_functions.py and analysis/common/lssph_b.py, plus numpy/scipy.
The fixtures it writes are committed; the tests read only the .npz files.

  kernels.npz   W(r, h) of the five kernels (KERNEL_TYPE 1..5) on a radius grid,
                from kernel_functions.{cubic_spline,quintic_spline,wendland_C2,
                wendland_C4,wendland_C6}_W
  lssph_b.npz   LS type-B (q = 3 and q = 6) interpolation of smooth fields at target
                points over a seeded jittered particle cloud, from lssph_b.main
                (analysis/common/lssph_b.py:21-143), the interpolation the reference
                uses for its virtual markers (interpolate_LSSPH_B_mod.f90)
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
    print("wrote", os.path.join(HERE, "kernels.npz"), os.path.join(HERE, "lssph_b.npz"))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
