"""Post-processing interpolation on the GPU: the reference's
``analysis/common/lssph_b.py`` ``main(param, target_x, target_y, x_j, y_j, val_j, rho_j)``
(LS-SPH type B, value and first derivatives at arbitrary points)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import Params, check

FIELDS = {"u": 0, "v": 1, "rho": 2, "pre": 3, "tem": 4}


def _d(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


_USED = ("h", "h_eff", "kernel_type", "sph_model", "target_problem", "SP_mass")


def _as_params(param) -> Params:
    """A Params as is; any other object (the analysis scripts' SimpleNamespace from
    read_utils) by the attributes the interpolation reads."""
    if isinstance(param, Params):
        return param
    p = Params()
    for name in _USED:
        setattr(p, name, getattr(param, name))
    return p


def lsb_interpolate(param, target_x, target_y, x_j, y_j, val_j, rho_j) -> np.ndarray:
    """Same arguments and result as the reference's ``lssph_b.main``: an (n_targets, 3) array
    of value, d/dx, d/dy, NaN where fewer than q particles lie within h_eff or the system is
    singular.  ``param`` is a Params or any object with h, h_eff, kernel_type, sph_model,
    target_problem and SP_mass."""
    param = _as_params(param)
    tx, ty, xs, ys, val, rho = (np.ascontiguousarray(a, dtype=np.float64).ravel()
                                for a in (target_x, target_y, x_j, y_j, val_j, rho_j))
    if tx.shape != ty.shape or not (xs.shape == ys.shape == val.shape == rho.shape):
        raise ValueError("target_x/target_y and x_j/y_j/val_j/rho_j must have matching lengths")
    out = np.empty((tx.shape[0], 3))
    check(_abi.load().lssph_lsb_interpolate(C.byref(param), xs.shape[0], _d(xs), _d(ys), _d(val), _d(rho),
                                            tx.shape[0], _d(tx), _d(ty), _d(out)))
    return out
