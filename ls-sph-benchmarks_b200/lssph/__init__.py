"""lssph -- Python host of the B200 LS-SPH engine (ctypes over include/lssph.h)."""
from ._abi import (LIB_PATH, PRECISION_FP64, PRECISION_MIXED, PRECISION_MIXED_COMPENSATED, LssphError, Params,
                   exported_names, load)
from .params import (boussinesq_params, cavity_params, check_param, default_params, diffusion_params,
                     from_config, init_param, make_params, taylor_green_params, write_config_h)
from .simulation import Simulation, State, estimate_device_bytes, read_data, setup_particles
from .batch import Batch
from .serving import Request, Server, ServerStats, device_memory
from .postproc import lsb_interpolate

__all__ = [
    "LIB_PATH", "PRECISION_FP64", "PRECISION_MIXED", "PRECISION_MIXED_COMPENSATED", "LssphError", "Params", "exported_names", "load",
    "boussinesq_params", "cavity_params", "check_param", "default_params", "diffusion_params",
    "from_config", "init_param", "make_params", "taylor_green_params", "write_config_h",
    "Simulation", "State", "estimate_device_bytes", "read_data", "setup_particles", "Batch",
    "Request", "Server", "ServerStats", "device_memory", "lsb_interpolate",
]
