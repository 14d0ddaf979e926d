"""ctypes wrapper of the CPU oracle (oracle/lssph_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the checker,
and by bench.py's CPU-baseline leg.  The engine never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liblssph_oracle.so")


class Params(C.Structure):
    """The oracle's own mirror of ``lssph_params`` (include/lssph.h, which the oracle's C++
    is compiled against): Param_type of source/core/global_types.f90:22-73 plus the
    boundary-code macros of config.h.  Defined here so that the checker and the CPU
    baseline never load the engine library; ``load()`` checks the size against the
    compiled struct."""

    _fields_ = [
        ("target_problem", C.c_int32),
        ("u_bc_top", C.c_int32), ("u_bc_bottom", C.c_int32), ("u_bc_left", C.c_int32), ("u_bc_right", C.c_int32),
        ("tem_bc_top", C.c_int32), ("tem_bc_bottom", C.c_int32), ("tem_bc_left", C.c_int32),
        ("tem_bc_right", C.c_int32),
        ("u_top", C.c_double), ("tem_top", C.c_double), ("tem_bottom", C.c_double), ("tem_left", C.c_double),
        ("tem_right", C.c_double),
        ("save_name", C.c_char * 256), ("read_name", C.c_char * 256),
        ("omp_threads", C.c_int32), ("rk", C.c_int32),
        ("len_x", C.c_double), ("len_y", C.c_double),
        ("num_x", C.c_int32), ("num_y", C.c_int32),
        ("start_step", C.c_int32), ("end_step", C.c_int32), ("write_step", C.c_int32), ("pad0_", C.c_int32),
        ("threshold", C.c_double), ("coe_CFL", C.c_double), ("coe_dif", C.c_double), ("zeta_RSST", C.c_double),
        ("xi_VIM", C.c_double),
        ("rho_ref", C.c_double), ("vis_ref", C.c_double), ("K_ref", C.c_double), ("k_th_ref", C.c_double),
        ("cp_ref", C.c_double), ("alpha_ref", C.c_double), ("gravity", C.c_double), ("pos_pert", C.c_double),
        ("tg_a", C.c_int32), ("tg_b", C.c_int32),
        ("coe_h", C.c_double), ("PST_c", C.c_double), ("coe_delta_sph", C.c_double),
        ("kernel_type", C.c_int32), ("sph_model", C.c_int32), ("wall_model", C.c_int32),
        ("total_step", C.c_int32), ("num_WL", C.c_int32), ("pad1_", C.c_int32),
        ("dx", C.c_double), ("SP_mass", C.c_double), ("h", C.c_double), ("h_eff", C.c_double),
        ("W_ave", C.c_double), ("WL_thick", C.c_double), ("delta_tem", C.c_double), ("tem_ave", C.c_double),
        ("sound_speed", C.c_double), ("kinematic_vis", C.c_double), ("thermal_dif", C.c_double),
        ("Re", C.c_double), ("Ra", C.c_double), ("Pr", C.c_double),
        ("dt", C.c_double), ("dt_CFL", C.c_double), ("dt_vis", C.c_double), ("dt_th", C.c_double),
        ("dt_CFL_relax", C.c_double), ("dt_vis_relax", C.c_double),
        ("precision", C.c_int32), ("lanes", C.c_int32), ("seed", C.c_uint64), ("periodic", C.c_int32),
        ("pad2_", C.c_int32),
    ]

    # config.h macro names -> fields (the engine-side extensions keep their field names)
    MACROS = {
        "TARGET_PROBLEM": "target_problem", "U_BOUNDARY_TOP": "u_bc_top", "U_BOUNDARY_BOTTOM": "u_bc_bottom",
        "U_BOUNDARY_LEFT": "u_bc_left", "U_BOUNDARY_RIGHT": "u_bc_right", "TEM_BOUNDARY_TOP": "tem_bc_top",
        "TEM_BOUNDARY_BOTTOM": "tem_bc_bottom", "TEM_BOUNDARY_LEFT": "tem_bc_left",
        "TEM_BOUNDARY_RIGHT": "tem_bc_right", "U_TOP": "u_top", "TEM_TOP": "tem_top", "TEM_BOTTOM": "tem_bottom",
        "TEM_LEFT": "tem_left", "TEM_RIGHT": "tem_right", "SAVE_NAME": "save_name", "READ_NAME": "read_name",
        "OMP_THREADS": "omp_threads", "LEN_X": "len_x", "LEN_Y": "len_y", "NUM_X": "num_x", "NUM_Y": "num_y",
        "RK": "rk", "START_STEP": "start_step", "END_STEP": "end_step", "WRITE_STEP": "write_step",
        "THRESHOLD": "threshold", "COE_CFL": "coe_CFL", "COE_DIF": "coe_dif", "ZETA_RSST": "zeta_RSST",
        "XI_VIM": "xi_VIM", "RHO_REF": "rho_ref", "VIS_REF": "vis_ref", "K_REF": "K_ref", "K_TH_REF": "k_th_ref",
        "CP_REF": "cp_ref", "ALPHA_REF": "alpha_ref", "GRAVITY": "gravity", "POS_PERT": "pos_pert",
        "TG_A": "tg_a", "TG_B": "tg_b", "COE_H": "coe_h", "PST_C": "PST_c", "COE_DELTA_SPH": "coe_delta_sph",
        "KERNEL_TYPE": "kernel_type", "SPH_MODEL": "sph_model", "WALL_MODEL": "wall_model", "PERIODIC": "periodic",
    }

    def copy(self) -> "Params":
        out = Params()
        C.memmove(C.byref(out), C.byref(self), C.sizeof(Params))
        return out

    def as_dict(self) -> dict:
        return {name: (getattr(self, name).decode() if isinstance(getattr(self, name), bytes) else getattr(self, name))
                for name, _ in self._fields_ if not name.startswith("pad")}


def as_params(p) -> Params:
    """An oracle Params with the bytes of ``p`` (any ctypes structure with the lssph_params
    layout, e.g. the engine binding's, as the tests pass them)."""
    if isinstance(p, Params):
        return p
    if C.sizeof(p) != C.sizeof(Params):
        raise TypeError(f"not an lssph_params layout: {C.sizeof(p)} bytes vs {C.sizeof(Params)}")
    out = Params()
    C.memmove(C.byref(out), C.byref(p), C.sizeof(Params))
    return out

_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int32)
_S = C.c_void_p
_PROTOS = {
    "orc_last_error": (C.c_char_p, []),
    "orc_set_threads": (C.c_int, [C.c_int]),
    "orc_init_param": (C.c_int, [C.POINTER(Params)]),
    "orc_params_default": (C.c_int, [C.POINTER(Params)]),
    "orc_params_sizeof": (C.c_size_t, []),
    "orc_kernel_W": (C.c_double, [C.c_int, C.c_double, C.c_double]),
    "orc_kernel_dW": (C.c_double, [C.c_int, C.c_double, C.c_double]),
    "orc_dgesv": (C.c_int, [C.c_int, C.c_int, _d, _d]),
    "orc_create_new": (_S, [C.POINTER(Params), C.c_int]),
    "orc_create_from": (_S, [C.POINTER(Params), C.c_int, C.c_int, _i, _d, _d, _d, _d, _d, _d, _d, C.c_int]),
    "orc_destroy": (None, [_S]),
    "orc_error": (C.c_int, [_S]),
    "orc_sizes": (C.c_int, [_S, _i, _i, _i, _i, _i]),
    "orc_get": (C.c_int, [_S, _i, _d, _d, _d, _d, _d, _d, _d]),
    "orc_set": (C.c_int, [_S, _d, _d, _d, _d, _d, _d, _d]),
    "orc_get_rhs": (C.c_int, [_S, _d, _d, _d, _d]),
    "orc_get_vm": (C.c_int, [_S, _i, _d, _d, _d, _d, _d, _d, _d, _d]),
    "orc_get_cells": (C.c_int, [_S, _i, _i]),
    "orc_calculate_rhs": (C.c_int, [_S]),
    "orc_update_cell": (C.c_int, [_S]),
    "orc_ghost": (C.c_int, [_S]),
    "orc_rk2": (C.c_int, [_S]),
    "orc_rk4": (C.c_int, [_S]),
    "orc_pst": (C.c_int, [_S]),
    "orc_check_steady_state": (C.c_int, [_S, _i]),
    "orc_run": (C.c_int, [_S, C.c_int, _i]),
    "orc_neighbors_csr": (C.c_int64, [_S, C.c_int, _i, _i, C.c_int64]),
    "orc_lssph_b": (C.c_int, [C.POINTER(Params), C.c_int, C.c_int, _d, _d, _d, _d, C.c_int, _d, _d, _d]),
    "orc_lsb_post": (C.c_int, [C.POINTER(Params), C.c_int, _d, _d, _d, _d, C.c_int, _d, _d, _d]),
}

_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            import importlib.util
            spec = importlib.util.spec_from_file_location("oracle_build", os.path.join(HERE, "build.py"))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            mod.build()
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if lib.orc_params_sizeof() != C.sizeof(Params):
            raise RuntimeError(f"oracle Params mirror is {C.sizeof(Params)} bytes, the compiled struct "
                               f"{lib.orc_params_sizeof()}")
        _lib = lib
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(_d)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_i)


def set_threads(n: int) -> int:
    return load().orc_set_threads(int(n))


def init_param(p) -> Params:
    q = as_params(p).copy()
    load().orc_init_param(C.byref(q))
    return q


def params_default() -> Params:
    """The reference's shipped config.h, derived (orc_params_default)."""
    p = Params()
    load().orc_params_default(C.byref(p))
    return p


def make_params(base: Params | None = None, **overrides) -> Params:
    """Copy ``base`` (default: config.h), set fields by config.h macro or field name, then
    derive (init_param_mod.f90:92-199).  The same overrides give the same bytes as the
    engine binding's ``lssph.make_params`` (checked in tests/test_oracle.py)."""
    p = (base or params_default()).copy()
    for k, v in overrides.items():
        name = Params.MACROS.get(k, k)
        if not hasattr(p, name):
            raise KeyError(f"unknown parameter {k}")
        setattr(p, name, v.encode() if isinstance(v, str) else v)
    load().orc_init_param(C.byref(p))
    return p


def taylor_green_params(num: int = 128, re: float = 100.0, coe_cfl: float = 0.1, tg: int = 2,
                        end_step: int = 12800, **kw) -> Params:
    """Problem 2 (Taylor-Green), RK4 + PST, VIS_REF = 1/Re: the same overrides as the
    engine binding's preset of that name."""
    return make_params(TARGET_PROBLEM=2, U_BOUNDARY_TOP=1, U_BOUNDARY_BOTTOM=1, U_BOUNDARY_LEFT=1,
                       U_BOUNDARY_RIGHT=1, NUM_X=num, NUM_Y=num, RK=4, VIS_REF=1.0 / re, K_REF=100.0,
                       COE_CFL=coe_cfl, TG_A=tg, TG_B=tg, PST_C=1.5, COE_DELTA_SPH=0.0, END_STEP=end_step,
                       **kw)


def kernel_W(kt: int, r: float, h: float) -> float:
    return load().orc_kernel_W(kt, r, h)


def kernel_dW(kt: int, r: float, h: float) -> float:
    return load().orc_kernel_dW(kt, r, h)


def dgesv(A: np.ndarray, B: np.ndarray) -> tuple[np.ndarray, int]:
    """Solve A X = B with the oracle's DGESV restatement (A, B not modified)."""
    n = A.shape[0]
    a = np.asfortranarray(A, dtype=np.float64).copy(order="F")
    b = np.asfortranarray(B.reshape(n, -1), dtype=np.float64).copy(order="F")
    info = load().orc_dgesv(n, b.shape[1], a.ctypes.data_as(_d), b.ctypes.data_as(_d))
    return b.reshape(B.shape), info


def lssph_b(p, q: int, xs, ys, rho, val, xt, yt) -> np.ndarray:
    p = as_params(p)
    xs, ys, rho, val, xt, yt = (np.ascontiguousarray(a, dtype=np.float64) for a in (xs, ys, rho, val, xt, yt))
    out = np.zeros(xt.shape[0])
    load().orc_lssph_b(C.byref(p), q, xs.shape[0], _dp(xs), _dp(ys), _dp(rho), _dp(val), xt.shape[0], _dp(xt),
                       _dp(yt), _dp(out))
    return out


def lsb_post(p, xt, yt, xs, ys, val, rho) -> np.ndarray:
    """analysis/common/lssph_b.py main(): (n_targets, 3) = value, d/dx, d/dy (NaN where
    fewer than q particles lie within h_eff or the system is singular)."""
    p = as_params(p)
    xs, ys, val, rho, xt, yt = (np.ascontiguousarray(a, dtype=np.float64) for a in (xs, ys, val, rho, xt, yt))
    out = np.zeros((xt.shape[0], 3))
    load().orc_lsb_post(C.byref(p), xs.shape[0], _dp(xs), _dp(ys), _dp(val), _dp(rho), xt.shape[0], _dp(xt),
                        _dp(yt), out.ctypes.data_as(_d))
    return out


class OracleError(RuntimeError):
    pass


class Oracle:
    """One CPU solve; the methods are the reference subroutines."""

    def __init__(self, p, state=None, num_int: int | None = None, ghost: bool = True):
        self._lib = load()
        self.params = as_params(p).copy()
        self.has_tem = p.target_problem == 4
        if state is None:
            self._s = self._lib.orc_create_new(C.byref(self.params), 1 if ghost else 0)
        else:
            pt = np.ascontiguousarray(state.ptype, dtype=np.int32)
            arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
                    (state.x, state.y, state.u, state.v, state.rho, state.pre)]
            tem = np.ascontiguousarray(state.tem, dtype=np.float64) if state.tem is not None else None
            self._s = self._lib.orc_create_from(C.byref(self.params), pt.shape[0], int(num_int), _ip(pt),
                                                *(_dp(a) for a in arrs), _dp(tem), 1 if ghost else 0)
        nt, ni, ne, nc, cap = (C.c_int32() for _ in range(5))
        self._lib.orc_sizes(self._s, *(C.byref(v) for v in (nt, ni, ne, nc, cap)))
        self.num_total, self.num_int, self.num_ext, self.num_cells, self.list_cap = (
            v.value for v in (nt, ni, ne, nc, cap))
        self._check()

    def _check(self, rc: int | None = None):
        err = self._lib.orc_error(self._s)
        if err:
            raise OracleError(f"[{err}] {self._lib.orc_last_error().decode()}")

    def close(self):
        if getattr(self, "_s", None):
            self._lib.orc_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get(self) -> dict:
        n = self.num_total
        out = {"ptype": np.zeros(n, np.int32), **{k: np.zeros(n) for k in ("x", "y", "u", "v", "rho", "pre", "tem")}}
        self._lib.orc_get(self._s, _ip(out["ptype"]), *(_dp(out[k]) for k in ("x", "y", "u", "v", "rho", "pre", "tem")))
        return out

    def set(self, **fields):
        arrs = {k: (np.ascontiguousarray(fields[k], dtype=np.float64) if k in fields else None)
                for k in ("x", "y", "u", "v", "rho", "pre", "tem")}
        self._lib.orc_set(self._s, *(_dp(arrs[k]) for k in ("x", "y", "u", "v", "rho", "pre", "tem")))

    def rhs(self) -> dict:
        n = self.num_int
        out = {k: np.zeros(n) for k in ("u", "v", "rho", "tem")}
        self._lib.orc_get_rhs(self._s, *(_dp(out[k]) for k in ("u", "v", "rho", "tem")))
        return out

    def vm(self) -> dict:
        n = self.num_ext
        out = {"ptype": np.zeros(n, np.int32),
               **{k: np.zeros(n) for k in ("x", "y", "u", "v", "pre", "tem", "nx", "ny")}}
        self._lib.orc_get_vm(self._s, _ip(out["ptype"]),
                             *(_dp(out[k]) for k in ("x", "y", "u", "v", "pre", "tem", "nx", "ny")))
        return out

    def cells(self) -> tuple[np.ndarray, np.ndarray]:
        a = np.zeros(self.num_total, np.int32)
        b = np.zeros(self.num_ext, np.int32)
        self._lib.orc_get_cells(self._s, _ip(a), _ip(b))
        return a, b

    def calculate_rhs(self):
        self._lib.orc_calculate_rhs(self._s); self._check()

    def update_cell(self):
        self._lib.orc_update_cell(self._s); self._check()

    def ghost(self):
        self._lib.orc_ghost(self._s); self._check()

    def rk2(self):
        self._lib.orc_rk2(self._s); self._check()

    def rk4(self):
        self._lib.orc_rk4(self._s); self._check()

    def pst(self):
        self._lib.orc_pst(self._s); self._check()

    def check_steady_state(self) -> bool:
        v = C.c_int32()
        self._lib.orc_check_steady_state(self._s, C.byref(v))
        return bool(v.value)

    def run(self, nsteps: int) -> int:
        v = C.c_int32()
        self._lib.orc_run(self._s, int(nsteps), C.byref(v))
        self._check()
        return v.value

    def neighbors(self, which: int = 0) -> tuple[np.ndarray, np.ndarray]:
        n = self.num_int if which == 0 else self.num_ext
        off = np.zeros(n + 1, np.int32)
        cap = n * 9 * max(self.list_cap, 1)
        idx = np.zeros(cap, np.int32)
        nnz = self._lib.orc_neighbors_csr(self._s, which, _ip(off), _ip(idx), cap)
        if nnz < 0:
            raise OracleError("neighbour buffer too small")
        return off, idx[:nnz]
