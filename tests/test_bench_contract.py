"""The benchmark's output contract and its multi-rank plumbing, on the CPU.

bench.py --impl reference times the CPU oracle on the headline workload and prints one
JSON line with the keys the engine's line carries; under torchrun only rank 0 prints.  The
engine arm takes the device time as the maximum over ranks, checked here with the gloo
backend on two CPU ranks.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _json_lines(out):
    return [json.loads(l) for l in out.splitlines() if l.strip().startswith("{")]


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "2", "--warmup", "3"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    d = lines[0]
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 3
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["config"]["workload"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["cores"] >= 1 and cb["kind"] in ("port", "reference") and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_never_loads_the_engine_library():
    # the reference arm builds its parameters with the oracle alone: no lssph module and no
    # liblssph.so mapping in its process
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '3']\n"
            "try:\n    runpy.run_path('bench.py', run_name='__main__')\nexcept SystemExit:\n    pass\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('ENGINE_SO', 'liblssph.so' in maps, 'ORACLE_SO', 'liblssph_oracle.so' in maps,"
            " 'LSSPH_MODULE', any(m == 'lssph' or m.startswith('lssph.') for m in sys.modules))\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "ENGINE_SO False ORACLE_SO True LSSPH_MODULE False" in r.stdout, r.stdout[-2000:]


def test_both_arms_report_the_same_config():
    # the oracle's parameter builder gives the engine's bytes, and both lines carry one dict
    sys.path.insert(0, ROOT)
    import bench
    import lssph
    import oracle as O
    pe, po = bench._params(), bench._oracle_params()
    assert bytes(pe) == bytes(O.as_params(pe)) and bytes(po) == bytes(O.as_params(pe))
    for kw in ({}, {"PERIODIC": 0}, {"num": 64, "re": 400.0}):
        a = lssph.taylor_green_params(**{**bench.HEADLINE, **{k: v for k, v in kw.items() if k != "PERIODIC"}},
                                      PERIODIC=kw.get("PERIODIC", 1))
        b = O.taylor_green_params(**{**bench.HEADLINE, **{k: v for k, v in kw.items() if k != "PERIODIC"}},
                                  PERIODIC=kw.get("PERIODIC", 1))
        assert bytes(a) == bytes(b), kw
    assert bytes(lssph.default_params()) == bytes(O.params_default())
    assert bench._config(pe, 16384, 16384) == bench._config(po, 16384, 16384)


def test_reference_arm_under_torchrun_prints_once():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1 and lines[0]["n_gpus"] == 2


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        q.put((rank, bench.max_over_ranks(1.5 + rank, dist, device="cpu")))
    finally:
        dist.destroy_process_group()


def test_device_time_is_the_maximum_over_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=5) for _ in procs)
    assert got == {0: 2.5, 1: 2.5}
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, None) == 3.25
