"""The validation runs at the benchmark problems' own horizons (lssph.validation), FP64 and
mixed precision side by side, checked on the CPU from their committed results file
(tests/golden/validation_results.json, written on one B200 by the command in
tests/golden/validation_results.cmd):

  * lid-driven cavity Re = 1000, 256^2 to t = 50: the centre-line profiles against the
    Ghia et al. (1982) table, read in place from the reference checkout as
    analysis/benchmarks/cavity_flow.py:41-55 reads it (skipped without LSSPH_REFERENCE_ROOT),
    and mixed precision against FP64;
  * Boussinesq Ra = 1e5: the bottom and top Nusselt numbers and their balance
    (analysis/benchmarks/boussinesq_conv.py:100-111), mixed against FP64;
  * periodic Taylor-Green to t = 1: the velocity error against the analytic decay and the
    kinetic-energy ratio against exp(-16 pi^2 nu t), mixed against FP64.
"""
import json
import os

import numpy as np
import pytest

from lssph import validation

HERE = os.path.dirname(os.path.abspath(__file__))
RESULTS = os.path.join(HERE, "golden", "validation_results.json")


@pytest.fixture(scope="module")
def results():
    if not os.path.exists(RESULTS):
        pytest.skip("no validation results committed")
    with open(RESULTS) as f:
        return json.load(f)["validation"]


def test_cavity_reaches_a_steady_state(results):
    for prec, r in results["cavity"].items():
        assert r["t_end"] == pytest.approx(50.0, rel=1e-6)
        v = np.array([h[1] for h in r["vrms_history"]])
        # V_rms over the last tenth of the run changes by less than 1 % of itself
        tail = v[int(0.9 * len(v)):]
        assert (tail.max() - tail.min()) < 0.01 * tail.mean(), prec


def test_cavity_profiles_mixed_equal_fp64(results):
    # at t = 50 the runs are far past the sensitivity horizon (the particle arrangements of
    # any two runs that differ in rounding have decorrelated), so the profiles agree to the
    # particle-noise level: measured 1.1e-2 (u) and 1.5e-2 (v) of the lid speed at most
    a, b = results["cavity"]["fp64"], results["cavity"]["mixed"]
    for k in ("u_at_x_half", "v_at_y_half"):
        assert np.max(np.abs(np.array(a[k]) - np.array(b[k]))) < 0.03, k


def test_cavity_profiles_against_ghia(results, reference_root):
    csv = os.path.join(reference_root, "analysis", "benchmarks", "Ghia_1982_Re_1000.csv")
    dev = validation.compare({"cavity": results["cavity"]}, csv)
    for prec, d in dev.items():
        # the reference's own error norms (cavity_flow.py:117-133), per precision; measured
        # L2 8.8e-2 / 9.1e-2 (u) and 1.1e-2 / 8.7e-3 (v, FP64 / mixed) at 256^2
        assert d["u"]["L2"] < 0.1 and d["v"]["L2"] < 0.05, (prec, d)
    # mixed precision moves the deviation from the literature by less than 1e-2 of the lid
    # speed (measured 2.9e-3 for u, 2.4e-3 for v)
    for c in ("u", "v"):
        assert abs(dev["mixed"][c]["L2"] - dev["fp64"][c]["L2"]) < 1e-2


def test_boussinesq_nusselt_balance(results):
    for prec, r in results["boussinesq"].items():
        assert r["nu_bottom"] > 1.0 and r["nu_top"] > 1.0, prec   # convecting, not conducting
        assert r["energy_balance_error_pct"] < 5.0, prec
        assert r["max_mach"] < 0.1, prec
    a, b = results["boussinesq"]["fp64"], results["boussinesq"]["mixed"]
    assert abs(a["nu_bottom"] - b["nu_bottom"]) < 0.02 * a["nu_bottom"]


def test_taylor_green_decay_to_t1(results):
    a, b = results["taylor_green"]["fp64"], results["taylor_green"]["mixed"]
    for r in (a, b):
        assert r["t_end"] == pytest.approx(1.0, rel=1e-9)
        assert r["velocity_rel_l2_vs_analytic"] < 0.05
        assert r["ke_ratio"] == pytest.approx(r["ke_ratio_exact"], rel=0.05)
    # the analytic-solution error is the same in both precisions (within 5 % of itself)
    assert abs(a["velocity_rel_l2_vs_analytic"] - b["velocity_rel_l2_vs_analytic"]) <= \
        0.05 * a["velocity_rel_l2_vs_analytic"]
