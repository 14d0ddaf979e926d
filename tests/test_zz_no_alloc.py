"""lssph_rhs_noalloc: the allocation-free RHS entry point, for callers that cannot
allocate GPU memory at the point of the call (all of their device memory is already
committed to their own pool, or the call sits in a loop where a driver allocation is not
acceptable).  The caller owns the state and output arrays on the device; the entry point
works in a static device array and must give the same RHS as the regular entry point
(lssph_calculate_rhs on a simulation handle).

The file name sorts last so that a run that stops at the first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

import lssph
import oracle as O
from lssph import _abi

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "u", "v", "rho", "pre")


def _device(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _rhs_noalloc(p, state, num_int, expect=0):
    """One lssph_rhs_noalloc call on device copies of `state`; returns host RHS arrays
    (or None when the call is expected to fail with status `expect`)."""
    import torch
    lib = lssph.load()
    n = state.num_total
    dev = [_device(getattr(state, k)) for k in FIELDS]
    tem = _device(state.tem) if p.target_problem == 4 else None
    outs = [torch.full((num_int,), np.nan, dtype=torch.float64, device="cuda") for _ in range(4)]
    torch.cuda.synchronize()
    rc = lib.lssph_rhs_noalloc(C.byref(p), n, num_int, *(t.data_ptr() for t in dev),
                               tem.data_ptr() if tem is not None else None,
                               outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(),
                               outs[3].data_ptr() if tem is not None else None, None)
    assert rc == expect, lib.lssph_last_error().decode()
    torch.cuda.synchronize()
    if expect:
        return None
    return {k: o.cpu().numpy() for k, o in zip(("u", "v", "rho", "tem"), outs)}


def _check(ref, got, keys):
    # same tolerance as the engine's lanes = 4 parity tests: 1e-12 of the field scale
    for k in keys:
        scale = max(np.abs(ref[k]).max(), 1e-30)
        assert np.abs(got[k] - ref[k]).max() <= 1e-12 * scale, k


def test_noalloc_rhs_matches_regular_entry_point_on_consecutive_calls():
    p = lssph.taylor_green_params(num=48, lanes=4)
    sim = lssph.Simulation.new(p)
    sim.step(2)
    # first call
    a = sim.download()
    sim.calculate_rhs()
    _check(sim.rhs(), _rhs_noalloc(p, a, sim.num_int), ("u", "v", "rho"))
    # second call, on a different state: the shared scratch must not carry anything over
    sim.step(3)
    b = sim.download()
    sim.calculate_rhs()
    _check(sim.rhs(), _rhs_noalloc(p, b, sim.num_int), ("u", "v", "rho"))


def test_noalloc_rhs_with_temperature():
    p = lssph.boussinesq_params(num=40, ra=1e5, lanes=4)
    sim = lssph.Simulation.new(p)
    sim.step(2)
    s = sim.download()
    sim.calculate_rhs()
    _check(sim.rhs(), _rhs_noalloc(p, s, sim.num_int), ("u", "v", "rho", "tem"))


def test_noalloc_rejects_sizes_beyond_its_limit():
    lib = lssph.load()
    p = lssph.taylor_green_params(num=32)
    too_many = 262144 + 1
    rc = lib.lssph_rhs_noalloc(C.byref(p), too_many, 1024, *([None] * 6), None, *([None] * 4), None)
    assert rc == _abi.E_BAD_PARAM   # null buffers are refused first
    fake = C.c_void_p(256)          # never dereferenced: the size check comes before any GPU work
    rc = lib.lssph_rhs_noalloc(C.byref(p), too_many, 1024, *([fake] * 6), None, *([fake] * 3), None, None)
    assert rc == _abi.E_CAPACITY
    assert b"262144" in lib.lssph_last_error()


def test_noalloc_rhs_with_one_lane_is_the_oracle_bit_for_bit():
    # lanes = 1 sums each particle's neighbours in the reference list order, so the RHS
    # equals the CPU restatement of calculate_RHS (LSSPH_A_mod.f90:26-271) bit for bit
    p = lssph.taylor_green_params(num=40, lanes=1)
    sim = lssph.Simulation.new(p)
    sim.step(3)
    s = sim.download()
    ni = sim.num_int
    sim.close()
    orc = O.Oracle(p, s, ni, ghost=False)
    orc.calculate_rhs()
    ref = orc.rhs()
    got = _rhs_noalloc(p, s, ni)
    for k in ("u", "v", "rho"):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


def test_noalloc_reports_cell_overflow_and_recovers():
    # more interior particles in one cell than its 32 slots: the scatter stops at the slot
    # limit (a bounds check before the write) and the call returns the overflow error; the
    # next call clears the shared counters and is correct again
    p = lssph.taylor_green_params(num=40, lanes=4)
    sim = lssph.Simulation.new(p)
    sim.step(1)
    good = sim.download()
    sim.calculate_rhs()
    ref = sim.rhs()
    ni = sim.num_int
    sim.close()
    bad = lssph.State(good.ptype, *(getattr(good, k).copy() for k in FIELDS))
    xc, yc = bad.x[ni // 2], bad.y[ni // 2]
    bad.x[:40] = xc
    bad.y[:40] = yc
    _rhs_noalloc(p, bad, ni, expect=_abi.E_CELL_OVERFLOW)
    assert b"particles in a cell" in lssph.load().lssph_last_error()
    _check(ref, _rhs_noalloc(p, good, ni), ("u", "v", "rho"))


def test_noalloc_reports_a_particle_outside_the_grid():
    # an interior particle far outside the box gets no cell key (checked before any list
    # write) and the call returns the out-of-domain error
    p = lssph.taylor_green_params(num=40, lanes=4)
    sim = lssph.Simulation.new(p)
    s = sim.download()
    ni = sim.num_int
    sim.close()
    s.x[7] = -5.0
    _rhs_noalloc(p, s, ni, expect=_abi.E_OUT_OF_DOMAIN)
    assert b"outside the cell grid" in lssph.load().lssph_last_error()
