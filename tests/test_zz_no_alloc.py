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
from lssph import _abi

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "u", "v", "rho", "pre")


def _device(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _rhs_noalloc(p, state, num_int):
    """One lssph_rhs_noalloc call on device copies of `state`; returns host RHS arrays."""
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
    assert rc == 0, lib.lssph_last_error().decode()
    torch.cuda.synchronize()
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
