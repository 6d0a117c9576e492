"""PANDORA 2.0 RK3 time step on B200 (sm_100a): host package over libpandora_gpu.so."""
from ._lib import PandoraError, device_count, lib_path, load  # noqa: F401
from .params import (NS_BF_ROT, NS_R_CONV, NS_R_ROT, PREC_FP32_MIXED, PREC_FP64, RK3_TIMESTEP_CFL,  # noqa: F401
                     RK3_TIMESTEP_DECIDE, RK3_TIMESTEP_FIXED, VISCOUS_EXPLICIT, VISCOUS_INTEGRATING_FACTOR, Params,
                     default_params, read_namelist, workload_params)
from .rk3 import (Simulation, ProgramInit, f_FluidstatsFs, f_InitialiseInit, f_RK3Stage1,  # noqa: F401
                  f_RK3Stage2, f_RK3Stage3, g_RK3Calc, p_ControlInitialiseParticles)
from .batch import Batch, batch_bytes, class_key  # noqa: F401
