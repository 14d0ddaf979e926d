"""The config.h parameter surface (source/setup/init_param_mod.f90,
source/check/check_param_mod.f90) as ``lssph_params`` structures."""
from __future__ import annotations

import ctypes as C

from . import _abi
from ._abi import Params, check


def default_params() -> Params:
    """Values of the reference's shipped config.h, with derived fields filled."""
    p = Params()
    check(_abi.load().lssph_params_default(C.byref(p)))
    return p


def from_config(path: str) -> Params:
    """Parse a config.h, derive (init_param) and validate (check_param)."""
    p = Params()
    check(_abi.load().lssph_params_from_config(str(path).encode(), C.byref(p)))
    return p


def init_param(p: Params) -> Params:
    check(_abi.load().lssph_init_param(C.byref(p)))
    return p


def check_param(p: Params) -> None:
    check(_abi.load().lssph_check_param(C.byref(p)))


def make_params(base: Params | None = None, **overrides) -> Params:
    """Copy ``base`` (default: reference defaults), apply overrides by field name or by
    config.h macro name, then init_param + check_param."""
    p = (base or default_params()).copy()
    for k, v in overrides.items():
        name = Params.MACROS.get(k, k)
        if not hasattr(p, name):
            raise KeyError(f"unknown parameter {k}")
        if isinstance(v, str):
            v = v.encode()
        setattr(p, name, v)
    init_param(p)
    check_param(p)
    return p


def write_config_h(p: Params, path: str) -> None:
    """Write a config.h that reproduces the user fields of ``p``."""
    lines = []
    for macro, field in Params.MACROS.items():
        v = getattr(p, field)
        if isinstance(v, bytes):
            lines.append(f'#define {macro} "{v.decode()}"')
        elif isinstance(v, float):
            lines.append(f"#define {macro} {repr(float(v)).replace('e', 'd') if 'e' in repr(float(v)) else repr(float(v)) + 'd0'}")
        else:
            lines.append(f"#define {macro} {int(v)}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


# The workloads named by the benchmark configurations, as reference parameter sets.
def diffusion_params(num: int = 50, pos_pert: float = 0.05, coe_dif: float = 0.1, seed: int = 0,
                     end_step: int = 1000, bc: int = 2, bc_tb: int | None = None, bc_lr: int | None = None,
                     **kw) -> Params:
    """Problem 1 (diffusion test): closed box, source-driven, RK2, jittered lattice.
    ``bc`` sets all four U_BOUNDARY_* (1 Neumann, 2 Dirichlet); bc_tb / bc_lr override
    top+bottom / left+right."""
    tb = bc if bc_tb is None else bc_tb
    lr = bc if bc_lr is None else bc_lr
    return make_params(TARGET_PROBLEM=1, U_BOUNDARY_TOP=tb, U_BOUNDARY_BOTTOM=tb, U_BOUNDARY_LEFT=lr,
                       U_BOUNDARY_RIGHT=lr, NUM_X=num, NUM_Y=num, RK=2, COE_DIF=coe_dif, POS_PERT=pos_pert,
                       END_STEP=end_step, seed=seed, **kw)


def taylor_green_params(num: int = 128, re: float = 100.0, coe_cfl: float = 0.1, tg: int = 2,
                        end_step: int = 12800, **kw) -> Params:
    """Problem 2 (Taylor-Green vortex, free-slip box), RK4 + PST, VIS_REF = 1/Re."""
    return make_params(TARGET_PROBLEM=2, U_BOUNDARY_TOP=1, U_BOUNDARY_BOTTOM=1, U_BOUNDARY_LEFT=1,
                       U_BOUNDARY_RIGHT=1, NUM_X=num, NUM_Y=num, RK=4, VIS_REF=1.0 / re, K_REF=100.0,
                       COE_CFL=coe_cfl, TG_A=tg, TG_B=tg, PST_C=1.5, COE_DELTA_SPH=0.0, END_STEP=end_step,
                       **kw)


def cavity_params(num: int = 256, re: float = 1000.0, coe_cfl: float = 0.5, end_step: int = 256000,
                  **kw) -> Params:
    """Problem 3 (lid-driven cavity), RK4 + PST, U_TOP = 1, VIS_REF = 1/Re."""
    return make_params(TARGET_PROBLEM=3, U_BOUNDARY_TOP=3, U_BOUNDARY_BOTTOM=2, U_BOUNDARY_LEFT=2,
                       U_BOUNDARY_RIGHT=2, U_TOP=1.0, NUM_X=num, NUM_Y=num, RK=4, VIS_REF=1.0 / re,
                       K_REF=100.0, COE_CFL=coe_cfl, END_STEP=end_step, **kw)


def boussinesq_params(num: int = 64, ra: float = 1.0e5, pr: float = 0.71, coe_cfl: float = 0.5,
                      end_step: int = 1000, **kw) -> Params:
    """Problem 4 (bottom-heated convection), rho0 = 1, alpha g dT = 1 (ALPHA_REF 0.1,
    GRAVITY 10, T_bottom 1, T_top 0): nu = sqrt(Pr/Ra), kappa = 1/sqrt(Ra Pr)."""
    nu = (pr / ra) ** 0.5
    kappa = 1.0 / (ra * pr) ** 0.5
    cp = 1.0e3
    return make_params(TARGET_PROBLEM=4, U_BOUNDARY_TOP=2, U_BOUNDARY_BOTTOM=2, U_BOUNDARY_LEFT=2,
                       U_BOUNDARY_RIGHT=2, TEM_BOUNDARY_TOP=1, TEM_BOUNDARY_BOTTOM=1, TEM_BOUNDARY_LEFT=2,
                       TEM_BOUNDARY_RIGHT=2, TEM_TOP=0.0, TEM_BOTTOM=1.0, NUM_X=num, NUM_Y=num, RK=4,
                       VIS_REF=nu, K_REF=100.0, K_TH_REF=kappa * cp, CP_REF=cp, ALPHA_REF=0.1, GRAVITY=10.0,
                       COE_CFL=coe_cfl, END_STEP=end_step, **kw)
