"""Validation runs of the benchmark problems at their own horizons, with the figures the
reference's analysis scripts compute from its snapshots, for FP64 and mixed precision side
by side:

  cavity        lid-driven cavity, Re = 1000, 256^2, RK4 + PST, to t = 50: the V_rms history
                and the centre-line profiles u(y) at x = L/2 and v(x) at y = L/2 by LS type-B
                interpolation of the final state (analysis/benchmarks/cavity_flow.py:76-120).
                The profiles are reported at 1025 points of each line (fine enough to be
                interpolated at any literature coordinate); compare() measures them against
                a Ghia et al. (1982) table read in place, as cavity_flow.py:41-55 reads it.
  boussinesq    bottom-heated convection, Ra = 1e5, Pr = 0.71, 128^2: the V_rms and Mach
                histories and the Nusselt numbers of the bottom and top walls from dT/dy with
                their energy-balance error (analysis/benchmarks/boussinesq_conv.py:59-111).
  taylor_green  periodic Taylor-Green, Re = 100, 128^2, to t = 1: the velocity error against
                the analytic decay exp(-8 pi^2 nu t) and the kinetic-energy ratio against
                exp(-16 pi^2 nu t) (analysis/benchmarks/taylor_green.py:35,113-123).

    python -m lssph.validation [--which cavity,boussinesq,taylor_green] [--out results.json]
    python -m lssph.validation --compare results.json --ghia .../Ghia_1982_Re_1000.csv

The runs take minutes on one B200 (256,000 cavity steps per precision).
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import (PRECISION_FP64, PRECISION_MIXED, PRECISION_MIXED_COMPENSATED, Simulation, boussinesq_params,
               cavity_params, make_params, taylor_green_params)

PRECISIONS = {"fp64": PRECISION_FP64, "mixed": PRECISION_MIXED, "mixed_compensated": PRECISION_MIXED_COMPENSATED}
PROFILE_POINTS = 1025


def _vrms(st, ni):
    return float(np.sqrt(np.mean(st.u[:ni] ** 2 + st.v[:ni] ** 2)))


def _advance(sim, nsteps, every, on_sample):
    """Step nsteps in chunks of `every`, calling on_sample(steps_done) after each chunk."""
    done = 0
    while done < nsteps:
        k = min(every, nsteps - done)
        sim.step(k)
        done += k
        on_sample(done)


def cavity(precision: str = "fp64", num: int = 256, re: float = 1000.0, t_end: float = 50.0,
           samples: int = 100) -> dict:
    p = make_params(cavity_params(num=num, re=re), precision=PRECISIONS[precision])
    nsteps = int(round(t_end / p.dt))
    sim = Simulation.new(p)
    hist = []
    t0 = time.perf_counter()
    _advance(sim, nsteps, max(1, nsteps // samples),
             lambda n: hist.append((n * p.dt, _vrms(sim.download(), sim.num_int))))
    wall = time.perf_counter() - t0
    L = p.len_x
    s = np.linspace(0.0, L, PROFILE_POINTS)
    u_line = sim.interpolate("u", np.full_like(s, 0.5 * L), s)[:, 0]
    v_line = sim.interpolate("v", s, np.full_like(s, 0.5 * L))[:, 0]
    tune = sim.tuning()
    sim.close()
    return {"problem": "lid-driven cavity", "re": re, "num": num, "precision": precision, "dt": p.dt,
            "steps": nsteps, "t_end": nsteps * p.dt, "wall_s": wall, "lanes": tune["lanes"],
            "vrms_history": hist, "line": s.tolist(), "u_at_x_half": u_line.tolist(),
            "v_at_y_half": v_line.tolist(), "u_top": p.u_top}


def boussinesq(precision: str = "fp64", num: int = 128, ra: float = 1.0e5, pr: float = 0.71,
               t_end: float = 100.0, samples: int = 100) -> dict:
    p = make_params(boussinesq_params(num=num, ra=ra, pr=pr), precision=PRECISIONS[precision])
    nsteps = int(round(t_end / p.dt))
    c_eff = p.sound_speed / (p.zeta_RSST * p.xi_VIM)
    sim = Simulation.new(p)
    hist = []

    def sample(n):
        st = sim.download()
        sp = st.u[:sim.num_int] ** 2 + st.v[:sim.num_int] ** 2
        hist.append((n * p.dt, float(np.sqrt(np.mean(sp))), float(np.sqrt(np.max(sp)) / c_eff)))

    t0 = time.perf_counter()
    _advance(sim, nsteps, max(1, nsteps // samples), sample)
    wall = time.perf_counter() - t0
    # Nusselt numbers from dT/dy on the walls (boussinesq_conv.py:90-111)
    x = np.linspace(0.0, p.len_x, p.num_x)
    dtdy_bot = sim.interpolate("tem", x, np.zeros_like(x))[:, 2]
    dtdy_top = sim.interpolate("tem", x, np.full_like(x, p.len_y))[:, 2]
    grad_ref = -p.delta_tem / p.len_y
    nu_bot, nu_top = float(np.mean(dtdy_bot / grad_ref)), float(np.mean(dtdy_top / grad_ref))
    tune = sim.tuning()
    sim.close()
    return {"problem": "Boussinesq convection", "ra": ra, "pr": pr, "num": num, "precision": precision,
            "dt": p.dt, "steps": nsteps, "t_end": nsteps * p.dt, "wall_s": wall, "lanes": tune["lanes"],
            "vrms_mach_history": hist, "nu_bottom": nu_bot, "nu_top": nu_top,
            "energy_balance_error_pct": abs(nu_bot - nu_top) / abs(nu_bot) * 100.0,
            "max_mach": max(h[2] for h in hist)}


def taylor_green(precision: str = "fp64", num: int = 128, re: float = 100.0, t_end: float = 1.0,
                 samples: int = 20) -> dict:
    p = make_params(taylor_green_params(num=num, re=re, coe_cfl=0.1, tg=2, PERIODIC=1),
                    precision=PRECISIONS[precision])
    nsteps = int(round(t_end / p.dt))
    sim = Simulation.new(p, ghost=False)
    ni = sim.num_int
    st0 = sim.download()
    ke0 = float(np.sum(st0.u[:ni] ** 2 + st0.v[:ni] ** 2))
    hist = []

    def sample(n):
        st = sim.download()
        t = n * p.dt
        dec = np.exp(-8.0 * np.pi ** 2 * p.kinematic_vis * t)
        x, y = st.x[:ni], st.y[:ni]
        ue = np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) * dec
        ve = -np.cos(2 * np.pi * x) * np.sin(2 * np.pi * y) * dec
        err = np.sqrt((np.sum((st.u[:ni] - ue) ** 2) + np.sum((st.v[:ni] - ve) ** 2)) /
                      (np.sum(ue ** 2) + np.sum(ve ** 2)))
        ke = float(np.sum(st.u[:ni] ** 2 + st.v[:ni] ** 2)) / ke0
        hist.append((t, float(err), ke, float(np.exp(-16.0 * np.pi ** 2 * p.kinematic_vis * t))))

    t0 = time.perf_counter()
    _advance(sim, nsteps, max(1, nsteps // samples), sample)
    wall = time.perf_counter() - t0
    tune = sim.tuning()
    sim.close()
    return {"problem": "Taylor-Green vortex (periodic)", "re": re, "num": num, "precision": precision,
            "dt": p.dt, "steps": nsteps, "t_end": nsteps * p.dt, "wall_s": wall, "lanes": tune["lanes"],
            "history_t_velerr_ke_ke_exact": hist, "velocity_rel_l2_vs_analytic": hist[-1][1],
            "ke_ratio": hist[-1][2], "ke_ratio_exact": hist[-1][3]}


RUNS = {"cavity": cavity, "boussinesq": boussinesq, "taylor_green": taylor_green}


def run(which=("cavity", "boussinesq", "taylor_green"), precisions=("fp64", "mixed")) -> dict:
    out = {}
    for name in which:
        out[name] = {prec: RUNS[name](prec) for prec in precisions}
    return out


def ghia_table(path: str):
    """A Ghia et al. (1982) centre-line table as cavity_flow.py:45-55 reads it: columns
    y, u (at x = 1/2) and x, v (at y = 1/2) in units of the box side and the lid speed."""
    d = np.loadtxt(path, delimiter=",", skiprows=1)
    return d[:, 0], d[:, 1], d[:, 2], d[:, 3]


def compare(results: dict, ghia_csv: str) -> dict:
    """Deviation of each precision's centre-line profiles from the Ghia table: the L1, L2 and
    L_inf norms of |u_SPH - u_Ghia| / U_top over Ghia's points (cavity_flow.py:117-133), the
    SPH profile taken at Ghia's coordinates by cubic interpolation of the 1025-point line."""
    from scipy.interpolate import CubicSpline
    ry, ru, rx, rv = ghia_table(ghia_csv)
    out = {}
    for prec, r in results["cavity"].items():
        s = np.asarray(r["line"])
        L, U = s[-1], r["u_top"]
        u = CubicSpline(s, r["u_at_x_half"])(ry * L)
        v = CubicSpline(s, r["v_at_y_half"])(rx * L)
        eu, ev = np.abs(u - ru * U) / U, np.abs(v - rv * U) / U
        out[prec] = {"u": {"L1": float(eu.mean()), "L2": float(np.sqrt((eu ** 2).mean())), "Linf": float(eu.max())},
                     "v": {"L1": float(ev.mean()), "L2": float(np.sqrt((ev ** 2).mean())), "Linf": float(ev.max())}}
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--which", default="cavity,boussinesq,taylor_green")
    ap.add_argument("--precision", default="fp64,mixed")
    ap.add_argument("--out", default="-")
    ap.add_argument("--compare", help="a results file of an earlier run")
    ap.add_argument("--ghia", help="Ghia et al. (1982) table for the cavity's Re (read in place)")
    a = ap.parse_args(argv)
    if a.compare:
        with open(a.compare) as f:
            res = json.load(f)
        print(json.dumps(compare(res.get("validation", res), a.ghia), indent=1))
        return 0
    res = {"validation": run(tuple(a.which.split(",")), tuple(a.precision.split(",")))}
    text = json.dumps(res)
    if a.out == "-":
        print(text)
    else:
        with open(a.out, "w") as f:
            f.write(text + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
