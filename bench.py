"""Benchmark of the LS-SPH engine: particle-updates/s per RK step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Workload (one "step" = one full time step of the hot path: RK4 stages, ghost bookkeeping,
PST): Taylor-Green vortex, Re = 100, 128^2 particles on the periodic unit square, RK4 with
particle shifting, CFL 0.1, FP64 -- the reference's problem 2 with TG_A = TG_B = 2 as the
benchmark's configuration 2 states it (synthetic initial state generated by the setup code;
no dataset).  The same flow in the reference's free-slip closed box is the `closed_box`
section of the line.

value  : interior particles x K / device time of the K timed steps (CUDA events on the
         engine's stream; an L2 flush -- a 256 MB write, then a 256 MB read of another buffer --
         separates consecutive steps).
         With N > 1 each rank runs an independent replica; value is the sum over ranks
         computed from the max over ranks of the device time (weak scaling).
e2e    : the same metric through the C ABI with host buffers: every step uploads the
         particle state from pinned host memory, steps, and downloads it again, in one
         lssph_advance_host call.
reference arm: the CPU restatement of the reference (oracle/) on all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ls-sph-benchmarks_b200"))

METRIC = "particle-updates/s per RK step"
UNIT = "particle-updates/s"
WORKLOAD = "taylor_green_re100_128x128_periodic_rk4_pst_fp64"


# The headline workload's parameters: Taylor-Green, Re = 100, 128^2, RK4 + PST, CFL 0.1,
# TG_A = TG_B = 2.  periodic: the benchmark's periodic unit square (its u = -cos 2pi x
# sin 2pi y is the reference's sin 2pi x cos 2pi y moved by a quarter period, the same
# flow); else the reference's free-slip closed box.
HEADLINE = dict(num=128, re=100.0, coe_cfl=0.1, tg=2)


def _params(lanes: int = 0, periodic: bool = True):
    """The engine arm's parameters, built by the engine's host code."""
    import lssph
    return lssph.taylor_green_params(**HEADLINE, lanes=lanes, PERIODIC=1 if periodic else 0)


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


def _oracle_params(periodic: bool = True):
    """The CPU arms' parameters, built by the oracle alone (its config.h defaults and
    init_param restatement), so that the reference arm never loads the engine library."""
    return _oracle().taylor_green_params(**HEADLINE, PERIODIC=1 if periodic else 0)


def _config(p, num_int, num_total):
    """The workload, identical in both arms' lines (arm-specific settings go elsewhere)."""
    return {"workload": WORKLOAD, "problem": "taylor_green", "num_x": p.num_x, "num_y": p.num_y,
            "num_int": num_int, "num_total": num_total, "rk": p.rk, "pst": True, "re": 1.0 / p.vis_ref,
            "dt": p.dt, "precision": "fp64", "domain": "periodic unit square" if p.periodic else "closed box",
            "l2": "device arm: a 256 MB write, then a 256 MB read of another buffer, flushes L2 between "
                  "timed steps (no inputs and no dirty lines in L2 when a step starts); host arm: not applicable"}


# ---------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------
_REASONS = ["gpu_idle", "applications_clocks_setting", "sw_power_cap", "hw_slowdown", "sync_boost",
            "sw_thermal_slowdown", "hw_thermal_slowdown", "hw_power_brake_slowdown"]


class ClockSampler:
    """SM clock, max clock and clock-event reasons sampled every 10 ms while the timed
    region runs.  Reads NVML (the library nvidia-smi reports from); falls back to
    `nvidia-smi -lms 200` when the NVML binding is missing."""

    def __init__(self, device_index: int):
        self.dev = device_index
        self.rows = []            # (sm_mhz, max_mhz, reasons_bits)
        self._stop = threading.Event()
        self._thread = None
        self._nvml = None
        self._h = None
        self._proc = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        self._nvml = pynvml
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            return pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def _sample(self):
        nv, h = self._nvml, self._h
        try:
            reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        except AttributeError:
            reasons = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        self.rows.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                          float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)), int(reasons)))

    def _loop(self):
        while not self._stop.wait(0.01):
            try:
                self._sample()
            except Exception:
                return

    def _smi_loop(self):
        for line in self._proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            try:
                bits = int(parts[2], 16) if parts[2].startswith("0x") else int(parts[2])
                self.rows.append((float(parts[0]), float(parts[1]), bits))
            except (ValueError, IndexError):
                continue

    def __enter__(self):
        try:
            self._h = self._nvml_handle()
            self._sample()
            self._thread = threading.Thread(target=self._loop, daemon=True)
        except Exception:
            self._nvml = None
            try:
                self._proc = subprocess.Popen(
                    ["nvidia-smi", "-i", str(self.dev), "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active",
                     "--format=csv,noheader,nounits", "-lms", "200"],
                    stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self._thread = threading.Thread(target=self._smi_loop, daemon=True)
            except OSError:
                self._thread = None
        if self._thread:
            self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._nvml is not None:
            if self._thread:
                self._thread.join(timeout=1)
            try:
                self._sample()
            except Exception:
                pass
        elif self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        reasons = set()
        for _, _, bits in self.rows:
            for i, name in enumerate(_REASONS):
                if bits & (1 << i) and name != "gpu_idle":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": self.rows[-1][1],
                "reasons": sorted(reasons), "samples": len(self.rows),
                "source": "nvml" if self._nvml is not None else "nvidia-smi"}


# ---------------------------------------------------------------------------------------
def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x: float, dist, device: str = "cuda") -> float:
    """The largest x of all ranks (each rank passes its own device time); x itself when
    there is no process group."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _profile_traffic():
    """DRAM bytes per k_stage launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "k_stage_taylor_green_128_periodic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def _measured_peaks():
    """HBM copy bandwidth: the measured-peaks file when present, else the same STREAM-style
    copy measured here (torch copy_ of 1 Gi bf16 elements, read + write bytes, best of 10)."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    try:
        import torch
        n = 1 << 30
        a = torch.empty(n, dtype=torch.bfloat16, device="cuda")
        b = torch.empty_like(a)
        a.fill_(1.0)
        b.copy_(a)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = float("inf")
        for _ in range(10):
            e0.record()
            b.copy_(a)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1) * 1e-3)
        del a, b
        torch.cuda.empty_cache()
        return 2.0 * n * 2 / best / 1e9, "measured here (torch copy_ of 1 Gi bf16, best of 10)"
    except Exception:   # noqa: BLE001 - no device memory for the probe
        return 6650.0, "fallback"


def _fp64_peak():
    """Measured FP64 peak: cuBLAS DGEMM 8192^3 (2*N^3 flops), best of 5, CUDA events.  The
    measured-peaks file carries HBM and bf16 figures only, so the FP64 denominator is taken here."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c = torch.empty_like(a)
    torch.matmul(a, b, out=c)
    best = float("inf")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(5):
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def cpu_baseline(min_seconds: float = 10.0, max_steps: int = 2000) -> dict:
    """The oracle on all host cores for a bounded sample of the same workload."""
    O = _oracle()
    cores = O.set_threads(os.cpu_count() or 1)
    orc = O.Oracle(_oracle_params())
    orc.run(2)                       # warm-up
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps:
        orc.run(5)
        steps += 5
        if time.perf_counter() - t0 >= min_seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": orc.num_int * steps / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{steps} time steps of the same workload ({dt:.1f} s, oracle/ C++ restatement, "
                      f"OpenMP over {cores} threads)", "num_int": orc.num_int}


def run_reference(args) -> int:
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    O = _oracle()
    cores = O.set_threads(os.cpu_count() or 1)
    p = _oracle_params()
    orc = O.Oracle(p)
    orc.run(args.warmup)
    t0 = time.perf_counter()
    orc.run(args.steps)
    dt = time.perf_counter() - t0
    value = orc.num_int * args.steps / dt
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": _config(p, orc.num_int, orc.num_total),
            "arm": {"parallelism": f"host CPU, OpenMP over {cores} threads (rank 0 only)",
                    "library": "oracle/_build/liblssph_oracle.so"},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{args.steps} time steps after {args.warmup} warm-up steps"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------
# The other configurations of the metric, reported beside the headline number
# ---------------------------------------------------------------------------------------
def _jittered(p, seed, amp=0.05):
    """Fresh-start state with seeded uniform position jitter of +-amp dx (interior)."""
    import numpy as np

    import lssph
    st, ni = lssph.setup_particles(p)
    rng = np.random.default_rng(seed)
    if p.target_problem != 1:   # problem 1 applies POS_PERT in its own setup
        st.x[:ni] += amp * p.dx * (2 * rng.random(ni) - 1)
        st.y[:ni] += amp * p.dx * (2 * rng.random(ni) - 1)
    return st, ni


def bench_mixed(steps: int = 100, acc_steps: int = 500) -> dict:
    """Lid-driven cavity, Re = 1000, 256^2, RK4 + PST: FP64 vs mixed precision, and the
    per-field relative L2 of mixed against FP64 after acc_steps steps (same inputs)."""
    import numpy as np

    import lssph
    out = {"workload": "cavity_re1000_256x256_rk4_pst", "steps": steps,
           "l2": "inputs larger than L2 not required: per-step working set ~45 MB, warm"}
    states = {}
    # each precision at the lane count (2 or 4 per particle) that runs it faster here
    for name, prec in (("fp64", lssph.PRECISION_FP64), ("mixed", lssph.PRECISION_MIXED)):
        best = None
        for lanes in (4, 2):
            p = lssph.make_params(lssph.cavity_params(num=256, re=1000.0), precision=prec, lanes=lanes)
            sim = lssph.Simulation.new(p)
            sim.step(5)
            sim.step(steps)
            ms, _ = sim.last_step_stats()
            v = sim.num_int * steps / (ms * 1e-3)
            if best is None or v > best[0]:
                if best is not None:
                    best[2].close()
                best = (v, lanes, sim)
            else:
                sim.close()
        v, lanes, sim = best
        out[f"{name}_value"] = v
        out[f"{name}_lanes"] = lanes
        out[f"{name}_register_budget"] = sim.tuning()["register_budget"]
        out[f"{name}_shape"] = sim.tuning()["shape"]
        sim.step(acc_steps - 5 - steps)
        states[name] = (sim.download(), sim.num_int)
        sim.close()
    out["value"] = out["mixed_value"]
    out["unit"] = UNIT
    out["speedup_vs_fp64"] = out["mixed_value"] / out["fp64_value"]
    (g64, ni), (gmx, _) = states["fp64"], states["mixed"]
    out["rel_l2_vs_fp64"] = {k: float(np.linalg.norm(getattr(gmx, k)[:ni] - getattr(g64, k)[:ni]) /
                                      np.linalg.norm(getattr(g64, k)[:ni])) for k in ("x", "y", "u", "v", "rho", "pre")}
    out["rel_l2_after_steps"] = acc_steps
    return out


def bench_closed_box(steps: int = 300) -> dict:
    """The same Taylor-Green 128^2 workload in the reference's own free-slip closed box
    (wall ghosts and the overlapped ghost schedule): device particle-updates/s over
    `steps` steps of one lssph_step call (5 MB working set, L2-resident either way)."""
    import lssph
    p = _params(periodic=False)
    sim = lssph.Simulation.new(p)
    sim.step(5)
    sim.step(steps)
    ms, nl = sim.last_step_stats()
    out = {"workload": "taylor_green_re100_128x128_closed_box_rk4_pst_fp64", "steps": steps,
           "value": sim.num_int * steps / (ms * 1e-3), "unit": UNIT, "us_per_step": 1e3 * ms / steps,
           "num_int": sim.num_int, "num_total": sim.num_total, "schedule": sim.tuning()}
    sim.close()
    return out


def bench_variants(steps: int = 50, cpu_seconds: float = 2.0) -> dict:
    """The other operator variants (SPH_MODEL 1/2 classical SPH, 4/5/6 higher-order LS) on
    the headline Taylor-Green 128^2 RK4 + PST workload: device particle-updates/s, and
    the oracle on all host cores over a short sample of the same solve."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    import lssph
    cores = O.set_threads(os.cpu_count() or 1)
    out = {"workload": "taylor_green_re100_128x128_rk4_pst_fp64", "steps": steps, "models": {}}
    for name, kw in (("classical_sum", {"SPH_MODEL": 1}), ("classical_difference", {"SPH_MODEL": 2}),
                     ("ls_q5", {"SPH_MODEL": 3}), ("ls_q9", {"SPH_MODEL": 4}), ("ls_q14", {"SPH_MODEL": 5}),
                     ("ls_q20_quintic", {"SPH_MODEL": 6, "KERNEL_TYPE": 2})):
        p = lssph.taylor_green_params(num=128, **kw)
        sim = lssph.Simulation.new(p)
        sim.step(5)
        sim.step(steps)
        ms, _ = sim.last_step_stats()
        row = {"value": sim.num_int * steps / (ms * 1e-3), "us_per_step": 1e3 * ms / steps}
        sim.close()
        orc = O.Oracle(p)
        orc.run(1)
        n, t0 = 0, time.perf_counter()
        while n < 200:
            orc.run(1)
            n += 1
            if time.perf_counter() - t0 >= cpu_seconds:
                break
        row["cpu_value"] = orc.num_int * n / (time.perf_counter() - t0)
        row["cpu_steps"] = n
        row["speedup_vs_cpu"] = row["value"] / row["cpu_value"]
        out["models"][name] = row
    out["unit"] = UNIT
    out["cpu_cores"] = cores
    return out


def bench_postproc(reps: int = 5) -> dict:
    """Post-processing LS type-B interpolation (analysis/common/lssph_b.py): points/s through
    the C ABI with host arrays (lsb_interpolate, what the analysis scripts would call on a
    .dat snapshot) and from the device-resident state (Simulation.interpolate), against the
    oracle's restatement on all host cores."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    import lssph
    cores = O.set_threads(os.cpu_count() or 1)
    out = {"unit": "points/s", "cpu_cores": cores, "cases": {}}
    for name, p, field, grid in (
            ("cavity_256_centre_profiles_q3", lssph.cavity_params(num=256), "u", False),
            ("cavity_256_full_field_q3", lssph.cavity_params(num=256), "u", True),
            ("boussinesq_128_wall_gradients_q6", lssph.boussinesq_params(num=128), "tem", False),
            ("boussinesq_96_q21_quintic", lssph.boussinesq_params(num=96, SPH_MODEL=6, KERNEL_TYPE=2), "tem", False)):
        sim = lssph.Simulation.new(p)
        sim.step(5)
        st = sim.download()
        L, n = p.len_x, p.num_x
        s = np.linspace(0.0, L, n)
        if grid:
            gx, gy = np.meshgrid((np.arange(n) + 0.5) * (L / n), (np.arange(n) + 0.5) * (L / n))
            tx, ty = gx.ravel(), gy.ravel()
        elif field == "tem":
            tx, ty = np.concatenate([s, s]), np.concatenate([np.zeros(n), np.full(n, L)])
        else:
            tx, ty = np.concatenate([np.full(n, 0.5 * L), s]), np.concatenate([s, np.full(n, 0.5 * L)])
        xs, ys, val = st.x - p.WL_thick, st.y - p.WL_thick, getattr(st, field)
        lssph.lsb_interpolate(p, tx, ty, xs, ys, val, st.rho)
        t = []
        for _ in range(reps):
            t0 = time.perf_counter()
            res = lssph.lsb_interpolate(p, tx, ty, xs, ys, val, st.rho)
            t.append(time.perf_counter() - t0)
        td = []
        for _ in range(reps):
            t0 = time.perf_counter()
            sim.interpolate(field, tx, ty)
            td.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        ref = O.lsb_post(p, tx, ty, xs, ys, val, st.rho)
        tc = time.perf_counter() - t0
        ok = ~np.isnan(ref[:, 0])
        rel = float((np.abs(res[ok] - ref[ok]).max(axis=0) / np.abs(ref[ok]).max(axis=0)).max()) if ok.any() else 0.0
        out["cases"][name] = {"points": int(tx.shape[0]), "particles": int(xs.shape[0]),
                              "gpu_host_arrays_points_per_s": tx.shape[0] / float(np.median(t)),
                              "gpu_device_state_points_per_s": tx.shape[0] / float(np.median(td)),
                              "cpu_points_per_s": tx.shape[0] / tc,
                              "speedup_host_arrays_vs_cpu": tc / float(np.median(t)),
                              "max_rel_diff_vs_oracle": rel}
        sim.close()
    return out


def bench_snapshots(steps: int = 200, every: int = 10) -> dict:
    """Taylor-Green 256^2 RK4 + PST with a data/<step>.dat snapshot every `every` steps:
    wall time per step without snapshots, with lssph_write_data (download + write, the
    reference's synchronous write_data) and with lssph_write_data_async."""
    import shutil
    import tempfile

    import lssph
    p = lssph.taylor_green_params(num=256)
    out = {"workload": f"taylor_green_256x256_rk4_pst_fp64, snapshot every {every} steps", "steps": steps}
    root = tempfile.mkdtemp(prefix="lssph_snap_")
    try:
        for mode in ("none", "sync", "async"):
            sim = lssph.Simulation.new(p)
            sim.step(5)
            t0 = time.perf_counter()
            for k in range(0, steps, every):
                sim.step(every)
                if mode == "sync":
                    sim.write_data(root, k + every)
                elif mode == "async":
                    sim.write_data_async(root, k + every)
            sim.snapshot_wait()
            out[f"{mode}_ms_per_step"] = 1e3 * (time.perf_counter() - t0) / steps
            sim.close()
        out["snapshot_bytes"] = os.path.getsize(os.path.join(root, p.save_name.decode(), "data", f"{steps}.dat"))
    finally:
        shutil.rmtree(root, ignore_errors=True)
    out["async_overhead_vs_none"] = out["async_ms_per_step"] / out["none_ms_per_step"] - 1.0
    out["sync_overhead_vs_none"] = out["sync_ms_per_step"] / out["none_ms_per_step"] - 1.0
    return out


def batched_mix(seed: int = 4, n: int = 64, precision: int = 0):
    """64 solves: half diffusion, half Taylor-Green, on the periodic unit square as the
    single-solve configurations state them; lattice side uniform over
    {32,48,64,96,128,192,256}; Re log-uniform in [50, 1000]; jitter +-0.05 dx."""
    import numpy as np

    import lssph
    rng = np.random.default_rng(seed)
    sides = [32, 48, 64, 96, 128, 192, 256]
    specs = []
    for k in range(n):
        side = int(rng.choice(sides))
        re = float(np.exp(rng.uniform(np.log(50.0), np.log(1000.0))))
        s = int(rng.integers(1 << 30))
        if k % 2 == 0:
            p = lssph.diffusion_params(num=side, pos_pert=0.05, seed=s, PERIODIC=1)
        else:
            p = lssph.taylor_green_params(num=side, re=re, PERIODIC=1)
        specs.append((lssph.make_params(p, precision=precision), s))
    return specs


def bench_batched(steps: int = 20) -> dict:
    import lssph
    out = {"workload": "64 solves on the periodic unit square: 32 diffusion + 32 Taylor-Green, "
                       "sides {32..256}, Re log-uniform [50,1000]",
           "steps": steps, "l2": "batched working set > L2 (126 MB); sequential runs are L2-warm"}
    # 64 sequential plain-FP64 runs, one after the other
    seq_ms, seq_units = 0.0, 0
    for p, s in batched_mix(precision=lssph.PRECISION_FP64):
        st, ni = _jittered(p, s)
        sim = lssph.Simulation(p, st, ni)
        sim.ghost()
        sim.step(3)
        sim.step(steps)
        seq_ms += sim.last_step_stats()[0]
        seq_units += ni * steps
        sim.close()
    out["sequential_fp64_value"] = seq_units / (seq_ms * 1e-3)
    finals = {}
    for name, prec in (("batched_fp64", lssph.PRECISION_FP64), ("batched_mixed", lssph.PRECISION_MIXED)):
        sims = []
        units = 0
        with lssph.Batch() as b:
            for p, s in batched_mix(precision=prec):
                st, ni = _jittered(p, s)
                sim = lssph.Simulation(p, st, ni)
                sim.ghost()
                sims.append(sim)
                b.add(sim)
                units += ni
            b.step(3)
            b.step(steps)
            ms, launches = b.last_step_stats()
        out[f"{name}_value"] = units * steps / (ms * 1e-3)
        out[f"{name}_launches_per_step"] = launches // steps
        finals[name] = [(sim.download(), sim.num_int) for sim in sims]
        for sim in sims:
            sim.close()
    # every field of every member, mixed against FP64 after the same 3 + steps steps
    import numpy as np
    worst = {}
    for (g64, ni), (gmx, _) in zip(finals["batched_fp64"], finals["batched_mixed"]):
        for k in ("x", "y", "u", "v", "rho", "pre"):
            ref = getattr(g64, k)[:ni]
            den = np.linalg.norm(ref)
            if den > 0:
                worst[k] = max(worst.get(k, 0.0), float(np.linalg.norm(getattr(gmx, k)[:ni] - ref) / den))
    out["rel_l2_mixed_vs_fp64_worst_member"] = worst
    out["max_rel_l2_mixed_vs_fp64"] = max(worst.values()) if worst else None
    out["total_particles"] = units
    out["value"] = out["batched_mixed_value"]
    out["unit"] = UNIT
    out["speedup_vs_sequential_fp64"] = out["batched_mixed_value"] / out["sequential_fp64_value"]
    return out


def _perturbed_temperature(p, seed: int, amp: float = 1e-3):
    """Initial state builder: fresh start plus a seeded uniform T perturbation of +-amp."""
    def init():
        import numpy as np

        import lssph
        st, ni = lssph.setup_particles(p)
        st.tem[:ni] += amp * (2.0 * np.random.default_rng(seed).random(ni) - 1.0)
        return st
    return init


def serving_requests(seed: int = 5, rate: float = 20.0, window_s: float = 8.0, median_steps: int = 60):
    """Poisson arrivals; 50% bottom-heated Boussinesq (Ra log-uniform [1e4, 1e6], Pr 0.71,
    seeded initial T perturbation of amplitude 1e-3), 50% lid-driven cavity (Re log-uniform
    [100, 3200]); lattice side uniform over 64..384 in steps of 32; mixed precision.  The
    simulated time of every request is t_end = 20 scaled by one factor, chosen so that the
    median request runs median_steps steps."""
    import numpy as np

    import lssph
    from lssph import Request
    rng = np.random.default_rng(seed)
    t, reqs = 0.0, []
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > window_s:
            break
        side = int(rng.choice(np.arange(64, 385, 32)))
        if rng.random() < 0.5:
            ra = float(np.exp(rng.uniform(np.log(1e4), np.log(1e6))))
            p = lssph.make_params(lssph.boussinesq_params(num=side, ra=ra, pr=0.71), precision=lssph.PRECISION_MIXED)
            init, tag = _perturbed_temperature(p, int(rng.integers(1 << 30))), "boussinesq"
        else:
            re = float(np.exp(rng.uniform(np.log(100.0), np.log(3200.0))))
            p = lssph.make_params(lssph.cavity_params(num=side, re=re), precision=lssph.PRECISION_MIXED)
            init, tag = None, "cavity"
        reqs.append(Request(rid=len(reqs), params=p, nsteps=0, arrival=t, tag=tag, init=init))
    steps20 = np.array([20.0 / r.params.dt for r in reqs])
    scale = median_steps / float(np.median(steps20))
    for r, n20 in zip(reqs, steps20):
        r.nsteps = max(1, int(round(n20 * scale)))
    return reqs, scale


def _serving_request(rng, rid, t, sides, t_end):
    """One request of the configuration-5 mix: 50% bottom-heated Boussinesq (Ra
    log-uniform [1e4, 1e6], Pr 0.71, seeded T perturbation 1e-3), 50% lid-driven cavity (Re
    log-uniform [100, 3200]); side drawn from `sides`; mixed precision; run to t_end."""
    import numpy as np

    import lssph
    from lssph import Request
    side = int(rng.choice(sides))
    if rng.random() < 0.5:
        ra = float(np.exp(rng.uniform(np.log(1e4), np.log(1e6))))
        p = lssph.make_params(lssph.boussinesq_params(num=side, ra=ra, pr=0.71), precision=lssph.PRECISION_MIXED)
        init, tag = _perturbed_temperature(p, int(rng.integers(1 << 30))), "boussinesq"
    else:
        re = float(np.exp(rng.uniform(np.log(100.0), np.log(3200.0))))
        p = lssph.make_params(lssph.cavity_params(num=side, re=re), precision=lssph.PRECISION_MIXED)
        init, tag = None, "cavity"
    return Request(rid=rid, params=p, nsteps=max(1, int(round(t_end / p.dt))), arrival=t, tag=tag, init=init)


CAPACITY_SIDES = (32, 48, 64)


def serving_capacity(sides=CAPACITY_SIDES, steps: int = 300, seed: int = 6) -> dict:
    """Measured capacity of the batched engine on the unscaled request mix (t_end = 20)
    restricted to `sides`: 24 requests of the mix stepped together for `steps` steps give
    the sustained particle-steps/s; divided by the mean work of a request (interior
    particles x steps to t = 20, averaged over the mix) it gives requests/s."""
    import numpy as np

    import lssph
    rng = np.random.default_rng(seed)
    reqs = [_serving_request(rng, k, 0.0, sides, 20.0) for k in range(24)]
    sims = []
    with lssph.Batch() as b:
        for r in reqs:
            if r.init is not None:
                sim = lssph.Simulation(r.params, r.init(), lssph.setup_particles(r.params)[1])
                sim.ghost()
            else:
                sim = lssph.Simulation.new(r.params)
            sims.append(sim)
            b.add(sim)
        b.step(20)
        b.step(steps)
        ms, _ = b.last_step_stats()
    ps = sum(s.num_int for s in sims) * steps / (ms * 1e-3)
    for s in sims:
        s.close()
    work = []
    for k in range(400):
        r = _serving_request(rng, k, 0.0, sides, 20.0)
        work.append(lssph.setup_particles(r.params)[1] * r.nsteps)
    return {"particle_steps_per_s": ps, "mean_request_particle_steps": float(np.mean(work)),
            "requests_per_s": ps / float(np.mean(work))}


def bench_serving(capacity_window_s: float = 120.0) -> dict:
    """The configuration-5 stream twice: (1) scaled -- arrivals at 20/s for 8 s over sides
    64..384 with t_end scaled so the median request runs 60 steps; (2) real physics --
    unscaled t_end = 20 over sides 32..64, arrivals at 90 % of the measured capacity for
    `capacity_window_s` seconds, run until every request has finished."""
    import numpy as np

    from lssph import Server
    reqs, scale = serving_requests()
    srv = Server(max_active=64, chunk_steps=20, keep_results=False)
    st = srv.run(reqs)
    srv.close()
    out = {"scaled": _serving_record(st, reqs, scale)}
    if capacity_window_s > 0:
        cap = serving_capacity()
        rate = 0.9 * cap["requests_per_s"]
        rng = np.random.default_rng(7)
        t, creqs = 0.0, []
        while True:
            t += float(rng.exponential(1.0 / rate))
            if t > capacity_window_s:
                break
            creqs.append(_serving_request(rng, len(creqs), t, CAPACITY_SIDES, 20.0))
        srv = Server(max_active=64, chunk_steps=100, keep_results=False)
        st = srv.run(creqs)
        srv.close()
        rec = _serving_record(st, creqs, 1.0)
        rec["workload"] = (f"Poisson {rate:.2f}/s (90 % of the measured capacity) for {capacity_window_s:.0f} s; "
                           "50% Boussinesq Ra [1e4,1e6], 50% cavity Re [100,3200]; sides 32, 48, 64; "
                           "unscaled t_end = 20; mixed precision")
        rec["capacity"] = cap
        rec["arrival_rate_per_s"] = rate
        rec["steps_per_request_median"] = float(np.median([r.nsteps for r in creqs]))
        out["capacity"] = rec
    return out


def _serving_record(st, reqs, scale) -> dict:
    return {"workload": "Poisson 20/s for 8 s; 50% Boussinesq Ra [1e4,1e6], 50% cavity Re [100,3200]; "
                        "sides 64..384 step 32; mixed precision",
            "t_end_scale": scale, "t_end": 20.0 * scale, "requests": len(reqs), "completed": st.completed,
            "p50_s": st.p50_s, "p99_s": st.p99_s, "solves_per_s": st.solves_per_s,
            "particle_updates_per_s": st.particle_updates_per_s, "device_busy_s": st.device_ms * 1e-3,
            "makespan_s": st.makespan_s, "max_active": st.max_active, "batch_calls": st.batch_calls,
            "max_queue": st.max_queue, "mean_queue": st.mean_queue,
            "host_setup_s": st.host_create_s, "host_wait_s": st.wait_s, "host_retire_s": st.host_retire_s,
            "host_launch_s": st.host_launch_s, "host_join_s": st.host_join_s,
            "admission": "first fit by exact device footprint within 80% of free HBM, 64 slots"}


def run_engine(args) -> int:
    import numpy as np
    import torch

    import lssph

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    p = _params(lanes=args.lanes)
    st, ni = lssph.setup_particles(p)
    sim = lssph.Simulation(p, st, ni)
    sim.ghost()
    n_total = sim.num_total
    # L2 flush between timed steps: a 256 MB write, then a 256 MB read of another buffer, so
    # that a step starts with none of its inputs in L2 and no dirty flush lines to write back
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    flush_read = torch.ones(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    # mean in-radius neighbour count P (the per-pair work unit of the roofline)
    off, _ = sim.neighbors(0)
    mean_p = float(off[-1]) / ni

    sim.step(args.warmup)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    dev_ms, launches = 0.0, 0
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            flush_read.sum()
            torch.cuda.synchronize()
            sim.step(1)
            ms, nl = sim.last_step_stats()
            dev_ms += ms
            launches += nl
    torch.cuda.synchronize()
    if dist:
        dev_ms = max_over_ranks(dev_ms, dist)
        dist.barrier()
    value = ws * ni * args.steps / (dev_ms * 1e-3)

    # velocity error against the analytic decay exp(-8 pi^2 nu t) after the timed steps
    cur = sim.download()
    t_now = (args.warmup + args.steps) * p.dt
    dec = np.exp(-8.0 * np.pi ** 2 * p.kinematic_vis * t_now)
    xs, ys = cur.x[:ni] - p.WL_thick, cur.y[:ni] - p.WL_thick
    ue = np.sin(2 * np.pi * xs) * np.cos(2 * np.pi * ys) * dec
    ve = -np.cos(2 * np.pi * xs) * np.sin(2 * np.pi * ys) * dec
    l2_analytic = float(np.sqrt((np.sum((cur.u[:ni] - ue) ** 2) + np.sum((cur.v[:ni] - ve) ** 2)) /
                                (np.sum(ue ** 2) + np.sum(ve ** 2))))

    # ---- per-kernel device times (same launch sequence, un-graphed, events per launch) ----
    prof_steps = max(5, min(50, args.steps))
    prof = sim.step_profiled(prof_steps)
    stage_ms, stage_n = prof["stage"]
    stage_avg_s = stage_ms * 1e-3 / max(stage_n, 1)
    flops_per_launch = ni * (101.0 * mean_p + 315.0)           # LSSPH_A q = 5, nb = 4
    bytes_per_launch = ni * 300.0                               # per particle-stage, FP64 SoA
    hbm_peak, peak_src = _measured_peaks()
    achieved_gbs = bytes_per_launch / stage_avg_s / 1e9
    traffic = _profile_traffic()
    tune = sim.tuning()
    fp64_peak = _fp64_peak()
    fp64_achieved = flops_per_launch / stage_avg_s / 1e12
    f_frac, b_frac = fp64_achieved / fp64_peak, achieved_gbs / hbm_peak
    # roofline of the dominant kernel: max(F / F_peak, B / B_peak), reported in the unit of
    # the term that wins; the other term rides along
    fp64_term = {"achieved": fp64_achieved, "peak": fp64_peak, "unit": "TFLOP/s", "frac": f_frac,
                 "peak_source": "measured here: cuBLAS DGEMM 8192^3, best of 5 (the measured-peaks "
                                "file has no FP64 figure)",
                 "flops_per_launch": flops_per_launch, "mean_neighbours": mean_p}
    hbm_term = {"achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s", "frac": b_frac,
                "peak_source": peak_src, "algorithmic_bytes_per_launch": bytes_per_launch}
    win = fp64_term if f_frac >= b_frac else hbm_term
    roofline = {"bound": "fp64" if win is fp64_term else "hbm",
                "kernel": f"k_stage<NB=4,G={tune['lanes']},{tune['register_budget']} registers>",
                "achieved": win["achieved"], "peak": win["peak"], "unit": win["unit"], "frac": win["frac"],
                "traffic": traffic, "fp64": fp64_term, "hbm": hbm_term,
                "launch_avg_us": stage_avg_s * 1e6,
                "kernel_share": {k: v[0] for k, v in prof.items()}}

    # ---- end to end through the C ABI with pinned host buffers ----
    e2e_steps = max(5, min(200, args.steps))
    pinned = {k: torch.empty(n_total, dtype=torch.float64, pin_memory=True).numpy()
              for k in ("x", "y", "u", "v", "rho", "pre")}
    host = sim.download()
    for k in pinned:
        pinned[k][:] = getattr(host, k)
    hst = lssph.State(host.ptype, *(pinned[k] for k in ("x", "y", "u", "v", "rho", "pre")))
    torch.cuda.synchronize()
    # the same round trip as three calls (upload, step, download), each synchronising
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sim.upload(hst)
        sim.step(1)
        sim.download_into(hst)
    sep_s = time.perf_counter() - t0
    # the headline: lssph_advance_host, the same copies and step queued with one synchronisation
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sim.advance_host(hst, 1)
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, dist)
    sep_s = max_over_ranks(sep_s, dist)
    nbytes = 6 * n_total * 8
    e2e = {"value": ws * ni * e2e_steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": nbytes,
           "d2h_bytes_per_step": nbytes, "steps": e2e_steps,
           "path": "lssph_advance_host(1) per step (upload from page-locked host arrays, one step, "
                   "download into them, one synchronisation), wall clock",
           "separate_calls_value": ws * ni * e2e_steps / sep_s,
           "separate_calls_path": "lssph_upload + lssph_step(1) + lssph_download per step"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline()
    extras, configs = {}, {}
    if rank == 0 and ws == 1 and not args.no_extras:
        # detail sections first; the configurations the metric names (mixed precision,
        # batched, serving) last, so that the end of the line carries their figures
        extras["closed_box"] = bench_closed_box()
        extras["variants"] = bench_variants()
        extras["postproc"] = bench_postproc()
        extras["snapshots"] = bench_snapshots()
        configs["mixed"] = bench_mixed()
        configs["batched"] = bench_batched()
        configs["serving"] = bench_serving(args.serving_seconds)

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": _config(p, ni, n_total),
            "engine": {"parallelism": f"replicas{ws}", "lanes": tune["lanes"],
                       "register_budget": tune["register_budget"], "global_batch": ni * ws},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "particle_stages_per_s": value * p.rk,
            "velocity_rel_l2_vs_analytic": {"value": l2_analytic, "t": t_now,
                                            "steps": args.warmup + args.steps},
            "clocks": clocks.summary(), **extras, **configs}
    if configs:
        line["summary_configs"] = summarize_configs(configs)
    print(json.dumps(line), flush=True)
    return 0


def summarize_configs(c: dict) -> dict:
    """Compact figures of the mixed-precision, batched and serving configurations (the last
    key of the line)."""
    m, b, s = c.get("mixed", {}), c.get("batched", {}), c.get("serving", {})
    r3 = lambda x: None if x is None else float(f"{x:.3g}")   # noqa: E731
    out = {"unit": UNIT}
    if m:
        out["mixed_cavity256"] = {"fp64": r3(m["fp64_value"]), "mixed": r3(m["mixed_value"]),
                                  "speedup": r3(m["speedup_vs_fp64"]),
                                  "max_rel_l2_vs_fp64": r3(max(m["rel_l2_vs_fp64"].values())),
                                  "after_steps": m["rel_l2_after_steps"]}
    if b:
        out["batched_64"] = {"sequential_fp64": r3(b["sequential_fp64_value"]),
                             "batched_fp64": r3(b["batched_fp64_value"]),
                             "batched_mixed": r3(b["batched_mixed_value"]),
                             "speedup_mixed_vs_sequential_fp64": r3(b["speedup_vs_sequential_fp64"]),
                             "max_rel_l2_mixed_vs_fp64": r3(b.get("max_rel_l2_mixed_vs_fp64"))}
    for key, name in (("scaled", "serving_scaled"), ("capacity", "serving_real_physics")):
        if key in s:
            d = s[key]
            out[name] = {k: r3(d[k]) if isinstance(d[k], float) else d[k]
                         for k in ("t_end", "requests", "completed", "p50_s", "p99_s", "solves_per_s",
                                   "max_queue", "mean_queue") if k in d}
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--lanes", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed-precision, batched and serving configurations")
    ap.add_argument("--serving-seconds", type=float, default=120.0,
                    help="arrival window of the real-physics serving stream (0 skips it)")
    ap.add_argument("--validate", action="store_true",
                    help="only the validation runs of lssph.validation (minutes), as one JSON line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.validate:
        from lssph import validation
        print(json.dumps({"validation": validation.run()}), flush=True)
        return 0
    if args.impl == "reference":
        return run_reference(args)
    return run_engine(args)


if __name__ == "__main__":
    sys.exit(main())
