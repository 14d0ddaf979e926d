"""ctypes binding of include/lssph.h (the engine's C ABI).

The library is loaded from ``ls-sph-benchmarks_b200/lib/liblssph.so`` (built in-tree by
``ls-sph-benchmarks_b200/build.py``).  There is no fallback: if the library is missing the
import of this module succeeds but every call raises ``LssphError``.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
# LSSPH_LIB selects another build of the engine (e.g. a tuning variant)
LIB_PATH = os.environ.get("LSSPH_LIB") or os.path.join(os.path.dirname(_PKG), "lib", "liblssph.so")

OK = 0
E_BAD_PARAM = -1
E_CUDA = -2
E_CELL_OVERFLOW = -3
E_OUT_OF_DOMAIN = -4
E_NONFINITE = -5
E_SINGULAR = -6
E_IO = -7
E_CAPACITY = -8
E_TIMEOUT = -9
E_UNSUPPORTED = -10

KIND_NAMES = ("stage", "cellsort", "ghost", "pst", "other")

PRECISION_FP64 = 0
PRECISION_MIXED = 1
PRECISION_MIXED_COMPENSATED = 2


class LssphError(RuntimeError):
    """A non-zero status from the engine (the reference would `error stop`)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status
        self.message = message


class Params(C.Structure):
    """Mirror of ``lssph_params`` (Param_type of source/core/global_types.f90:22-73
    plus the boundary-code macros of config.h)."""

    _fields_ = [
        ("target_problem", C.c_int32),
        ("u_bc_top", C.c_int32), ("u_bc_bottom", C.c_int32),
        ("u_bc_left", C.c_int32), ("u_bc_right", C.c_int32),
        ("tem_bc_top", C.c_int32), ("tem_bc_bottom", C.c_int32),
        ("tem_bc_left", C.c_int32), ("tem_bc_right", C.c_int32),
        ("u_top", C.c_double),
        ("tem_top", C.c_double), ("tem_bottom", C.c_double),
        ("tem_left", C.c_double), ("tem_right", C.c_double),
        ("save_name", C.c_char * 256),
        ("read_name", C.c_char * 256),
        ("omp_threads", C.c_int32),
        ("rk", C.c_int32),
        ("len_x", C.c_double), ("len_y", C.c_double),
        ("num_x", C.c_int32), ("num_y", C.c_int32),
        ("start_step", C.c_int32), ("end_step", C.c_int32), ("write_step", C.c_int32),
        ("pad0_", C.c_int32),
        ("threshold", C.c_double), ("coe_CFL", C.c_double), ("coe_dif", C.c_double),
        ("zeta_RSST", C.c_double), ("xi_VIM", C.c_double),
        ("rho_ref", C.c_double), ("vis_ref", C.c_double), ("K_ref", C.c_double),
        ("k_th_ref", C.c_double), ("cp_ref", C.c_double), ("alpha_ref", C.c_double),
        ("gravity", C.c_double), ("pos_pert", C.c_double),
        ("tg_a", C.c_int32), ("tg_b", C.c_int32),
        ("coe_h", C.c_double), ("PST_c", C.c_double), ("coe_delta_sph", C.c_double),
        ("kernel_type", C.c_int32), ("sph_model", C.c_int32), ("wall_model", C.c_int32),
        ("total_step", C.c_int32), ("num_WL", C.c_int32),
        ("pad1_", C.c_int32),
        ("dx", C.c_double), ("SP_mass", C.c_double), ("h", C.c_double), ("h_eff", C.c_double),
        ("W_ave", C.c_double), ("WL_thick", C.c_double),
        ("delta_tem", C.c_double), ("tem_ave", C.c_double),
        ("sound_speed", C.c_double), ("kinematic_vis", C.c_double), ("thermal_dif", C.c_double),
        ("Re", C.c_double), ("Ra", C.c_double), ("Pr", C.c_double),
        ("dt", C.c_double), ("dt_CFL", C.c_double), ("dt_vis", C.c_double), ("dt_th", C.c_double),
        ("dt_CFL_relax", C.c_double), ("dt_vis_relax", C.c_double),
        ("precision", C.c_int32),
        ("lanes", C.c_int32),
        ("seed", C.c_uint64),
        ("periodic", C.c_int32),
        ("pad2_", C.c_int32),
    ]

    # user-facing names of config.h macros -> fields
    MACROS = {
        "TARGET_PROBLEM": "target_problem", "U_BOUNDARY_TOP": "u_bc_top",
        "U_BOUNDARY_BOTTOM": "u_bc_bottom", "U_BOUNDARY_LEFT": "u_bc_left",
        "U_BOUNDARY_RIGHT": "u_bc_right", "TEM_BOUNDARY_TOP": "tem_bc_top",
        "TEM_BOUNDARY_BOTTOM": "tem_bc_bottom", "TEM_BOUNDARY_LEFT": "tem_bc_left",
        "TEM_BOUNDARY_RIGHT": "tem_bc_right", "U_TOP": "u_top", "TEM_TOP": "tem_top",
        "TEM_BOTTOM": "tem_bottom", "TEM_LEFT": "tem_left", "TEM_RIGHT": "tem_right",
        "SAVE_NAME": "save_name", "READ_NAME": "read_name", "OMP_THREADS": "omp_threads",
        "LEN_X": "len_x", "LEN_Y": "len_y", "NUM_X": "num_x", "NUM_Y": "num_y", "RK": "rk",
        "START_STEP": "start_step", "END_STEP": "end_step", "WRITE_STEP": "write_step",
        "THRESHOLD": "threshold", "COE_CFL": "coe_CFL", "COE_DIF": "coe_dif",
        "ZETA_RSST": "zeta_RSST", "XI_VIM": "xi_VIM", "RHO_REF": "rho_ref", "VIS_REF": "vis_ref",
        "K_REF": "K_ref", "K_TH_REF": "k_th_ref", "CP_REF": "cp_ref", "ALPHA_REF": "alpha_ref",
        "GRAVITY": "gravity", "POS_PERT": "pos_pert", "TG_A": "tg_a", "TG_B": "tg_b",
        "COE_H": "coe_h", "PST_C": "PST_c", "COE_DELTA_SPH": "coe_delta_sph",
        "KERNEL_TYPE": "kernel_type", "SPH_MODEL": "sph_model", "WALL_MODEL": "wall_model",
        "PERIODIC": "periodic",
    }

    def copy(self) -> "Params":
        out = Params()
        C.memmove(C.byref(out), C.byref(self), C.sizeof(Params))
        return out

    def as_dict(self) -> dict:
        d = {}
        for name, _ in self._fields_:
            if name.startswith("pad"):
                continue
            v = getattr(self, name)
            d[name] = v.decode() if isinstance(v, bytes) else v
        return d


_P = C.POINTER
_d = _P(C.c_double)
_i = _P(C.c_int32)
_H = C.c_void_p

# name -> (restype, argtypes)
_PROTOS = {
    "lssph_abi_version": (C.c_int, []),
    "lssph_params_sizeof": (C.c_size_t, []),
    "lssph_last_error": (C.c_char_p, []),
    "lssph_status_string": (C.c_char_p, [C.c_int]),
    "lssph_params_default": (C.c_int, [_P(Params)]),
    "lssph_params_from_config": (C.c_int, [C.c_char_p, _P(Params)]),
    "lssph_init_param": (C.c_int, [_P(Params)]),
    "lssph_check_param": (C.c_int, [_P(Params)]),
    "lssph_setup_counts": (C.c_int, [_P(Params), _i, _i]),
    "lssph_setup_particles": (C.c_int, [_P(Params), C.c_int32, _i, _d, _d, _d, _d, _d, _d, _d]),
    "lssph_create": (C.c_int, [_P(Params), C.c_int32, C.c_int32, _i, _d, _d, _d, _d, _d, _d, _d,
                               _P(C.c_void_p)]),
    "lssph_destroy": (None, [_H]),
    "lssph_handle_error": (C.c_char_p, [_H]),
    "lssph_get_params": (C.c_int, [_H, _P(Params)]),
    "lssph_counts": (C.c_int, [_H, _i, _i, _i, _i]),
    "lssph_calculate_rhs": (C.c_int, [_H]),
    "lssph_update_cell": (C.c_int, [_H]),
    "lssph_ghost": (C.c_int, [_H]),
    "lssph_rk2": (C.c_int, [_H]),
    "lssph_rk4": (C.c_int, [_H]),
    "lssph_pst": (C.c_int, [_H]),
    "lssph_check_steady_state": (C.c_int, [_H, _i]),
    "lssph_step": (C.c_int, [_H, C.c_int32, _i]),
    "lssph_upload": (C.c_int, [_H, _d, _d, _d, _d, _d, _d, _d]),
    "lssph_download": (C.c_int, [_H, _i, _d, _d, _d, _d, _d, _d, _d]),
    "lssph_advance_host": (C.c_int, [_H, C.c_int32, _d, _d, _d, _d, _d, _d, _d, _i]),
    "lssph_download_rhs": (C.c_int, [_H, _d, _d, _d, _d]),
    "lssph_download_vm": (C.c_int, [_H, _i, _d, _d, _d, _d, _d, _d]),
    "lssph_neighbors_csr": (C.c_int, [_H, C.c_int32, _i, _i, C.c_int64, _P(C.c_int64)]),
    "lssph_write_data": (C.c_int, [_H, C.c_char_p, C.c_int32]),
    "lssph_write_param": (C.c_int, [_H, C.c_char_p, C.c_char_p]),
    "lssph_write_parameters": (C.c_int, [_P(Params), C.c_int32, C.c_int32, C.c_char_p]),
    "lssph_read_data": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, _i, _d, _d, _d, _d, _d, _d, _d]),
    "lssph_last_step_stats": (C.c_int, [_H, _P(C.c_double), _P(C.c_int64)]),
    "lssph_mem_info": (C.c_int, [_P(C.c_int64), _P(C.c_int64)]),
    "lssph_device_bytes": (C.c_int, [_H, _P(C.c_int64)]),
    "lssph_estimate_device_bytes": (C.c_int, [_P(Params), _P(C.c_int64)]),
    "lssph_set_step_budget": (C.c_int, [_H, C.c_int32]),
    "lssph_get_progress": (C.c_int, [_H, _i, _i]),
    "lssph_get_schedule": (C.c_int, [_H, _i, _i, _i]),
    "lssph_get_tuning": (C.c_int, [_H, _i, _i, _P(C.c_double), _P(C.c_double)]),
    "lssph_get_kernel_shape": (C.c_int, [_H, _i]),
    "lssph_step_profiled": (C.c_int, [_H, C.c_int32, _d, _P(C.c_int64)]),
    "lssph_batch_create": (C.c_int, [_P(C.c_void_p)]),
    "lssph_batch_destroy": (None, [_H]),
    "lssph_batch_error": (C.c_char_p, [_H]),
    "lssph_batch_add": (C.c_int, [_H, _H]),
    "lssph_batch_remove": (C.c_int, [_H, _H]),
    "lssph_batch_size": (C.c_int, [_H]),
    "lssph_batch_step": (C.c_int, [_H, C.c_int32, _i, _i, _i]),
    "lssph_batch_launch": (C.c_int, [_H, C.c_int32]),
    "lssph_batch_wait": (C.c_int, [_H, _i, _i, _i]),
    "lssph_batch_last_step_stats": (C.c_int, [_H, _P(C.c_double), _P(C.c_int64)]),
    "lssph_write_data_async": (C.c_int, [_H, C.c_char_p, C.c_int32]),
    "lssph_snapshot_wait": (C.c_int, [_H]),
    "lssph_lsb_interpolate": (C.c_int, [_P(Params), C.c_int32, _d, _d, _d, _d, C.c_int32, _d, _d, _d]),
    "lssph_interpolate": (C.c_int, [_H, C.c_int32, C.c_int32, _d, _d, _d]),
    # device pointers (caller-owned device memory), stream handle
    "lssph_rhs_noalloc": (C.c_int, [_P(Params), C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p]),
}

_lib = None


def exported_names() -> list:
    """Every symbol this binding expects the library to export."""
    return sorted(_PROTOS)


def load(path: str | None = None):
    """Load (once) and return the engine library with prototypes applied."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise LssphError(E_UNSUPPORTED,
                         f"engine library not built: {p} (run python ls-sph-benchmarks_b200/build.py)")
    lib = C.CDLL(p)
    for name, (res, args) in _PROTOS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.lssph_params_sizeof() != C.sizeof(Params):
        raise LssphError(E_BAD_PARAM, "lssph_params layout mismatch between library and binding")
    if path is None:
        _lib = lib
    return lib


def check(status: int, handle=None) -> int:
    if status == OK:
        return status
    lib = load()
    if handle:
        msg = lib.lssph_handle_error(handle)
    else:
        msg = lib.lssph_last_error()
    raise LssphError(status, (msg or b"").decode(errors="replace"))


def dptr(a):
    """Pointer to a contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(_d)


def iptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_i)
