"""ctypes wrapper of the CPU oracle (oracle/lssph_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the checker,
and by bench.py's CPU-baseline leg.  The engine never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "ls-sph-benchmarks_b200"))

from lssph._abi import Params  # noqa: E402  (shared struct layout of include/lssph.h)

LIB_PATH = os.path.join(HERE, "_build", "liblssph_oracle.so")

_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int32)
_S = C.c_void_p
_PROTOS = {
    "orc_last_error": (C.c_char_p, []),
    "orc_set_threads": (C.c_int, [C.c_int]),
    "orc_init_param": (C.c_int, [C.POINTER(Params)]),
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
        _lib = lib
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(_d)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_i)


def set_threads(n: int) -> int:
    return load().orc_set_threads(int(n))


def init_param(p: Params) -> Params:
    q = p.copy()
    load().orc_init_param(C.byref(q))
    return q


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


def lssph_b(p: Params, q: int, xs, ys, rho, val, xt, yt) -> np.ndarray:
    xs, ys, rho, val, xt, yt = (np.ascontiguousarray(a, dtype=np.float64) for a in (xs, ys, rho, val, xt, yt))
    out = np.zeros(xt.shape[0])
    load().orc_lssph_b(C.byref(p), q, xs.shape[0], _dp(xs), _dp(ys), _dp(rho), _dp(val), xt.shape[0], _dp(xt),
                       _dp(yt), _dp(out))
    return out


def lsb_post(p: Params, xt, yt, xs, ys, val, rho) -> np.ndarray:
    """analysis/common/lssph_b.py main(): (n_targets, 3) = value, d/dx, d/dy (NaN where
    fewer than q particles lie within h_eff or the system is singular)."""
    xs, ys, val, rho, xt, yt = (np.ascontiguousarray(a, dtype=np.float64) for a in (xs, ys, val, rho, xt, yt))
    out = np.zeros((xt.shape[0], 3))
    load().orc_lsb_post(C.byref(p), xs.shape[0], _dp(xs), _dp(ys), _dp(val), _dp(rho), xt.shape[0], _dp(xt),
                        _dp(yt), out.ctypes.data_as(_d))
    return out


class OracleError(RuntimeError):
    pass


class Oracle:
    """One CPU solve; the methods are the reference subroutines."""

    def __init__(self, p: Params, state=None, num_int: int | None = None, ghost: bool = True):
        self._lib = load()
        self.params = p.copy()
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
