"""Snapshots that do not stop the time loop (needs a B200).

lssph_write_data_async must write exactly the file lssph_write_data writes for the same
state (write_data_mod.f90:40-54 layout), while later steps proceed; a solve restarted from
such a file (restart_mod.f90 + lssph_create) must continue bit for bit like the solve that
never stopped, which is what checkpointing or pre-empting a running solve relies on.
"""
import os

import numpy as np
import pytest

import lssph

pytestmark = pytest.mark.gpu

CASES = {
    "diffusion": lambda: lssph.diffusion_params(num=40, seed=2),
    "taylor_green": lambda: lssph.taylor_green_params(num=48),
    "cavity": lambda: lssph.cavity_params(num=48),
    "boussinesq": lambda: lssph.boussinesq_params(num=40),
}


def _sim(p):
    st, ni = lssph.setup_particles(p)
    sim = lssph.Simulation(p, st, ni)
    sim.ghost()
    return sim


def _read(path):
    with open(path, "rb") as f:
        return f.read()


@pytest.mark.parametrize("case", list(CASES))
def test_async_files_equal_sync_files(case, tmp_path):
    p = CASES[case]()
    a, b = _sim(p), _sim(p)
    ra, rb = str(tmp_path / "a"), str(tmp_path / "b")
    for step in (5, 10, 15):
        a.step(5)
        a.write_data_async(ra, step)      # returns at once; stepping continues
        b.step(5)
        b.write_data(rb, step)
    a.step(3)                             # steps while the last file may still be written
    a.snapshot_wait()
    name = p.save_name.decode() if isinstance(p.save_name, bytes) else p.save_name
    for step in (5, 10, 15):
        fa = os.path.join(ra, name, "data", f"{step}.dat")
        fb = os.path.join(rb, name, "data", f"{step}.dat")
        assert _read(fa) == _read(fb), step
    a.close()
    b.close()


def test_close_waits_for_pending_snapshots(tmp_path):
    p = CASES["taylor_green"]()
    sim = _sim(p)
    sim.step(2)
    sim.write_data_async(str(tmp_path), 2)
    sim.close()
    name = p.save_name.decode() if isinstance(p.save_name, bytes) else p.save_name
    path = os.path.join(str(tmp_path), name, "data", "2.dat")
    assert os.path.getsize(path) == sim.num_total * (4 + 6 * 8)


def test_write_error_is_reported(tmp_path):
    p = CASES["cavity"]()
    sim = _sim(p)
    blocker = tmp_path / "file"
    blocker.write_text("not a directory")
    with pytest.raises(lssph.LssphError):
        sim.write_data_async(str(blocker), 1)    # results root is a file: no data/ directory
    sim.close()


@pytest.mark.parametrize("case", ["taylor_green", "cavity", "boussinesq"])
def test_restart_from_async_snapshot_is_bit_identical(case, tmp_path):
    p = CASES[case]()
    run = _sim(p)
    run.step(10)
    run.write_data_async(str(tmp_path), 10)
    run.step(10)                            # the uninterrupted solve, 20 steps
    run.snapshot_wait()
    name = p.save_name.decode() if isinstance(p.save_name, bytes) else p.save_name
    st = lssph.read_data(os.path.join(str(tmp_path), name, "data", "10.dat"), p)
    ni = run.num_int
    resumed = lssph.Simulation(p, st, ni)   # restart: state from the file, no extra ghost pass
    resumed.step(10)
    g, r = run.download(), resumed.download()
    for k in ("x", "y", "u", "v", "rho", "pre") + (("tem",) if p.target_problem == 4 else ()):
        assert np.array_equal(getattr(g, k), getattr(r, k)), k
    run.close()
    resumed.close()


@pytest.mark.parametrize("case", ["diffusion", "taylor_green", "cavity", "boussinesq", "tg_periodic", "tg_mixed",
                                  "cavity_classical"])
def test_upload_mid_run_continues_bit_identically(case):
    # lssph_upload into a solve at another point of its run (other buffer parity, other
    # list rotation): the state it continues from is the uploaded one, nothing else
    mk = dict(CASES)
    # lanes fixed: with lanes = 0 each handle of a periodic solve picks 2 or 4 by timing
    mk["tg_periodic"] = lambda: lssph.taylor_green_params(num=48, PERIODIC=1, lanes=4)
    mk["tg_mixed"] = lambda: lssph.make_params(lssph.taylor_green_params(num=48), precision=lssph.PRECISION_MIXED)
    mk["cavity_classical"] = lambda: lssph.cavity_params(num=40, SPH_MODEL=1)
    p = mk[case]()
    a, b = _sim(p), _sim(p)
    a.step(10)
    mid = a.download()
    a.step(10)
    b.step(3)                 # b is elsewhere in its run
    b.upload(mid)
    b.step(10)
    ga, gb = a.download(), b.download()
    for k in ("x", "y", "u", "v", "rho", "pre") + (("tem",) if p.target_problem == 4 else ()):
        assert np.array_equal(getattr(ga, k), getattr(gb, k)), k
    a.close()
    b.close()
