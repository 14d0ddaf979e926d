"""Host-side mirror of the reference's solver interface over the engine's C ABI.

The reference drives its solver from ``program main`` (source/main.f90:15-168) with
subroutines that act on Fortran derived types; the same operators are methods here:

=====================  ==============================================  ===================
reference subroutine   file:line                                       here
=====================  ==============================================  ===================
init_param             source/setup/init_param_mod.f90:24              params.init_param
check_param            source/check/check_param_mod.f90:22             params.check_param
init_particle          source/setup/init_particle_mod.f90:46           Simulation.new
restart_closed_box     source/setup/restart_mod.f90:22                 Simulation.restart
calculate_RHS          source/equation/calculate_RHS_mod.f90:29        .calculate_rhs
update_cell            source/neighbor/update_cell_mod.f90:21          .update_cell
ghost                  source/boundary/ghost_mod.f90:43                .ghost
RK2 / RK4              source/equation/RK2_mod.f90:30, RK4_mod.f90:30  .rk2 / .rk4
PST                    source/shifting/PST_mod.f90:28                  .pst
check_steady_state     source/check/check_steady_state_mod.f90:23      .check_steady_state
write_param            source/io/write_param_mod.f90:27                .write_param
write_data             source/io/write_data_mod.f90:22                 .write_data
time-loop body         source/main.f90:119-149                         .step(n)
=====================  ==============================================  ===================

Errors that make the reference ``error stop`` raise ``LssphError``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import LssphError, Params, check, dptr, iptr


@dataclass
class State:
    """SoA particle state in reference order (interior first, then ghosts)."""

    ptype: np.ndarray
    x: np.ndarray
    y: np.ndarray
    u: np.ndarray
    v: np.ndarray
    rho: np.ndarray
    pre: np.ndarray
    tem: np.ndarray | None = None

    @property
    def num_total(self) -> int:
        return int(self.x.shape[0])

    def copy(self) -> "State":
        return State(*(None if a is None else a.copy() for a in
                       (self.ptype, self.x, self.y, self.u, self.v, self.rho, self.pre, self.tem)))


def setup_particles(p: Params) -> tuple[State, int]:
    """setup_closed_box + impose_* initial conditions; returns (state, num_int)."""
    lib = _abi.load()
    nt = C.c_int32()
    ni = C.c_int32()
    check(lib.lssph_setup_counts(C.byref(p), C.byref(nt), C.byref(ni)))
    n = nt.value
    st = State(np.zeros(n, np.int32), *(np.zeros(n) for _ in range(6)),
               tem=np.zeros(n) if p.target_problem == 4 else None)
    check(lib.lssph_setup_particles(C.byref(p), n, iptr(st.ptype), dptr(st.x), dptr(st.y),
                                    dptr(st.u), dptr(st.v), dptr(st.rho), dptr(st.pre),
                                    dptr(st.tem)))
    return st, ni.value


def _c64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class Simulation:
    """One device-resident solve (an ``lssph_handle``)."""

    def __init__(self, params: Params, state: State, num_int: int):
        self._lib = _abi.load()
        self.params = params.copy()
        self.num_int = int(num_int)
        self.num_total = state.num_total
        self.num_ext = self.num_total - self.num_int
        self.has_tem = params.target_problem == 4
        h = C.c_void_p()
        pt = np.ascontiguousarray(state.ptype, dtype=np.int32)
        arrs = [_c64(a) for a in (state.x, state.y, state.u, state.v, state.rho, state.pre)]
        tem = _c64(state.tem) if self.has_tem else None
        check(self._lib.lssph_create(C.byref(self.params), self.num_total, self.num_int, iptr(pt),
                                     *(dptr(a) for a in arrs), dptr(tem), C.byref(h)))
        self._h = h
        self.ptype = pt.copy()

    # ---- construction ---------------------------------------------------------------
    @classmethod
    def new(cls, params: Params, ghost: bool = True) -> "Simulation":
        """Fresh start (init_particle with READ_NAME = "new"); ghost() as write_param does."""
        st, ni = setup_particles(params)
        sim = cls(params, st, ni)
        if ghost:
            sim.ghost()
        return sim

    @classmethod
    def restart(cls, params: Params, path: str) -> "Simulation":
        """restart_closed_box: read <step>.dat and continue from it."""
        st = read_data(path, params)
        _, ni = setup_particles(params)
        return cls(params, st, ni)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.lssph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _chk(self, status: int) -> int:
        return check(status, self._h)

    # ---- reference operators --------------------------------------------------------
    def calculate_rhs(self) -> None:
        self._chk(self._lib.lssph_calculate_rhs(self._h))

    def update_cell(self) -> None:
        self._chk(self._lib.lssph_update_cell(self._h))

    def ghost(self) -> None:
        self._chk(self._lib.lssph_ghost(self._h))

    def rk2(self) -> None:
        self._chk(self._lib.lssph_rk2(self._h))

    def rk4(self) -> None:
        self._chk(self._lib.lssph_rk4(self._h))

    def pst(self) -> None:
        self._chk(self._lib.lssph_pst(self._h))

    def check_steady_state(self) -> bool:
        s = C.c_int32()
        self._chk(self._lib.lssph_check_steady_state(self._h, C.byref(s)))
        return bool(s.value)

    def step(self, nsteps: int = 1) -> int:
        """Time-loop body for nsteps steps; returns the 1-based steady step or 0."""
        s = C.c_int32()
        self._chk(self._lib.lssph_step(self._h, int(nsteps), C.byref(s)))
        return s.value

    # ---- state transfer ---------------------------------------------------------------
    def download(self) -> State:
        n = self.num_total
        st = State(np.zeros(n, np.int32), *(np.zeros(n) for _ in range(6)),
                   tem=np.zeros(n) if self.has_tem else None)
        self._chk(self._lib.lssph_download(self._h, iptr(st.ptype), dptr(st.x), dptr(st.y), dptr(st.u),
                                           dptr(st.v), dptr(st.rho), dptr(st.pre), dptr(st.tem)))
        return st

    def download_into(self, st: State) -> None:
        self._chk(self._lib.lssph_download(self._h, None, dptr(st.x), dptr(st.y), dptr(st.u),
                                           dptr(st.v), dptr(st.rho), dptr(st.pre), dptr(st.tem)))

    def advance_host(self, st: State, nsteps: int = 1) -> int:
        """Upload ``st`` (positions and fields), run ``nsteps`` steps and write the new state
        back into ``st``'s arrays, with one synchronisation (lssph_advance_host).  The arrays
        must be C-contiguous float64 (page-locked ones are read and written in place by one
        kernel each way).  Returns the step at which problem 1 reached its steady state in
        this call, or 0."""
        for a in (st.x, st.y, st.u, st.v, st.rho, st.pre) + ((st.tem,) if self.has_tem else ()):
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.shape[0] != self.num_total:
                raise ValueError("advance_host needs C-contiguous float64 arrays of num_total entries")
        steady = C.c_int32()
        self._chk(self._lib.lssph_advance_host(self._h, int(nsteps), dptr(st.x), dptr(st.y), dptr(st.u),
                                               dptr(st.v), dptr(st.rho), dptr(st.pre),
                                               dptr(st.tem) if self.has_tem else None, C.byref(steady)))
        return steady.value

    def upload(self, st: State) -> None:
        arrs = [_c64(a) for a in (st.x, st.y, st.u, st.v, st.rho, st.pre)]
        tem = _c64(st.tem) if self.has_tem else None
        self._chk(self._lib.lssph_upload(self._h, *(dptr(a) for a in arrs), dptr(tem)))

    def rhs(self) -> dict:
        n = self.num_int
        out = {k: np.zeros(n) for k in ("u", "v", "rho", "tem")}
        self._chk(self._lib.lssph_download_rhs(self._h, dptr(out["u"]), dptr(out["v"]), dptr(out["rho"]),
                                               dptr(out["tem"])))
        if not self.has_tem:
            out.pop("tem")
        return out

    def virtual_markers(self) -> dict:
        n = self.num_ext
        out = {"ptype": np.zeros(n, np.int32), **{k: np.zeros(n) for k in ("x", "y", "u", "v", "pre", "tem")}}
        self._chk(self._lib.lssph_download_vm(self._h, iptr(out["ptype"]), dptr(out["x"]), dptr(out["y"]),
                                              dptr(out["u"]), dptr(out["v"]), dptr(out["pre"]), dptr(out["tem"])))
        return out

    def neighbors(self, which: int = 0) -> tuple[np.ndarray, np.ndarray]:
        """Sorted in-radius neighbour sets as CSR (offsets, indices)."""
        n = self.num_int if which == 0 else self.num_ext
        off = np.zeros(n + 1, np.int32)
        nnz = C.c_int64()
        self._chk(self._lib.lssph_neighbors_csr(self._h, which, iptr(off), None, 0, C.byref(nnz)))
        idx = np.zeros(max(nnz.value, 1), np.int32)
        self._chk(self._lib.lssph_neighbors_csr(self._h, which, iptr(off), iptr(idx), idx.size, C.byref(nnz)))
        return off, idx[: nnz.value]

    def step_profiled(self, nsteps: int = 1) -> dict:
        """Same launches as step(), un-graphed, with per-kernel CUDA events.  Returns
        {kind: (total_ms, launches)} for the kinds of _abi.KIND_NAMES."""
        ms = (C.c_double * len(_abi.KIND_NAMES))()
        nl = (C.c_int64 * len(_abi.KIND_NAMES))()
        self._chk(self._lib.lssph_step_profiled(self._h, int(nsteps), ms, nl))
        return {k: (ms[i], nl[i]) for i, k in enumerate(_abi.KIND_NAMES)}

    def interpolate(self, field: str, target_x, target_y) -> np.ndarray:
        """LS type-B value, d/dx, d/dy of ``field`` ("u", "v", "rho", "pre", "tem") at points
        of the analysis frame (positions minus WL_thick), from the current device state:
        the reference's lssph_b.main over a .dat snapshot, without the download."""
        from .postproc import FIELDS
        tx = np.ascontiguousarray(target_x, dtype=np.float64).ravel()
        ty = np.ascontiguousarray(target_y, dtype=np.float64).ravel()
        if tx.shape != ty.shape:
            raise ValueError("target_x and target_y must have the same length")
        out = np.empty((tx.shape[0], 3))
        dp = C.POINTER(C.c_double)
        self._chk(self._lib.lssph_interpolate(self._h, FIELDS[field], tx.shape[0], tx.ctypes.data_as(dp),
                                              ty.ctypes.data_as(dp), out.ctypes.data_as(dp)))
        return out

    def device_bytes(self) -> int:
        """Device memory this solve holds (requested bytes)."""
        n = C.c_int64()
        self._chk(self._lib.lssph_device_bytes(self._h, C.byref(n)))
        return n.value

    def set_step_budget(self, nsteps: int) -> None:
        """Stop advancing after nsteps more steps (0 removes the budget)."""
        self._chk(self._lib.lssph_set_step_budget(self._h, int(nsteps)))

    def progress(self) -> tuple[int, str]:
        """(steps completed since creation, "running" | "steady" | "budget")."""
        n, st = C.c_int32(), C.c_int32()
        self._chk(self._lib.lssph_get_progress(self._h, C.byref(n), C.byref(st)))
        return n.value, ("running", "steady", "budget")[st.value]

    def tuning(self) -> dict:
        """Kernel configuration picked for this solve (lanes, register budget, timings, and
        the tile schedule of the time step)."""
        lanes, tight = C.c_int32(), C.c_int32()
        lo, ti = C.c_double(), C.c_double()
        self._chk(self._lib.lssph_get_tuning(self._h, C.byref(lanes), C.byref(tight), C.byref(lo), C.byref(ti)))
        nt, ni, ov = C.c_int32(), C.c_int32(), C.c_int32()
        self._chk(self._lib.lssph_get_schedule(self._h, C.byref(nt), C.byref(ni), C.byref(ov)))
        shape = C.c_int32()
        self._chk(self._lib.lssph_get_kernel_shape(self._h, C.byref(shape)))
        return {"lanes": lanes.value, "register_budget": ("loose", "tight", "five", "six", "eight")[tight.value],
                "shape": ("fused", "split", "thread", "warp")[shape.value],
                "rhs_us_loose": lo.value, "rhs_us_tight": ti.value, "tiles": nt.value,
                "interior_tiles": ni.value, "ghost_overlap": bool(ov.value)}

    def last_step_stats(self) -> tuple[float, int]:
        ms = C.c_double()
        nl = C.c_int64()
        self._chk(self._lib.lssph_last_step_stats(self._h, C.byref(ms), C.byref(nl)))
        return ms.value, nl.value

    # ---- results/ files -----------------------------------------------------------------
    def write_param(self, results_root: str, config_h: str | None = None) -> None:
        self._chk(self._lib.lssph_write_param(self._h, results_root.encode(),
                                              (config_h or "").encode()))

    def write_data(self, results_root: str, step: int) -> None:
        self._chk(self._lib.lssph_write_data(self._h, results_root.encode(), int(step)))

    def write_data_async(self, results_root: str, step: int) -> None:
        """write_data that returns at once: the state is captured on the device and the file
        is written in the background while stepping continues (snapshot_wait to finish)."""
        self._chk(self._lib.lssph_write_data_async(self._h, results_root.encode(), int(step)))

    def snapshot_wait(self) -> None:
        """Wait for every pending write_data_async file of this solve."""
        self._chk(self._lib.lssph_snapshot_wait(self._h))


def setup_counts(params: Params) -> tuple[int, int]:
    """(num_total, num_int) of the closed box described by params."""
    lib = _abi.load()
    nt, ni = C.c_int32(), C.c_int32()
    check(lib.lssph_setup_counts(C.byref(params), C.byref(nt), C.byref(ni)))
    return nt.value, ni.value


def estimate_device_bytes(params: Params) -> int:
    """Device bytes Simulation.new(params) will allocate (host-side computation)."""
    lib = _abi.load()
    n = C.c_int64()
    check(lib.lssph_estimate_device_bytes(C.byref(params), C.byref(n)))
    return n.value


def read_data(path: str, params: Params) -> State:
    """Read a results/<name>/data/<step>.dat snapshot (write_data_mod.f90:40-54)."""
    lib = _abi.load()
    nt = C.c_int32()
    ni = C.c_int32()
    check(lib.lssph_setup_counts(C.byref(params), C.byref(nt), C.byref(ni)))
    n = nt.value
    with_tem = params.target_problem == 4
    st = State(np.zeros(n, np.int32), *(np.zeros(n) for _ in range(6)),
               tem=np.zeros(n) if with_tem else None)
    check(lib.lssph_read_data(path.encode(), n, 1 if with_tem else 0, iptr(st.ptype), dptr(st.x), dptr(st.y),
                              dptr(st.u), dptr(st.v), dptr(st.rho), dptr(st.pre), dptr(st.tem)))
    return st


__all__ = ["State", "Simulation", "setup_particles", "read_data", "LssphError"]
