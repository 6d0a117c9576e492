"""ctypes binding of libpandora_gpu.so (the C-ABI of include/pandora_gpu.h).

The library is built in-tree (``python pandora-2.0_b200/build.py``) and loaded
from this package's parent directory.  There is no CPU fallback: if the shared
library or a CUDA device is missing, the calls that need them raise.
"""
from __future__ import annotations

import ctypes
import os

from .params import Params

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "libpandora_gpu.so")

OK = 0
ERR_INVALID_ARG = -1
ERR_OOM = -2
ERR_CUDA = -3
ERR_NAN = -4
ERR_TIMEOUT = -5
ERR_BAD_LAYOUT = -6
ERR_CFL = -7
ERR_PARTICLE_LOST = -8
ERR_NO_DEVICE = -9
ERR_UNSUPPORTED = -10


class PandoraError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {msg} (status {status})")
        self.status = status


_lib = None
_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64

# name -> argtypes (restype int unless listed in _RESTYPES)
SIGNATURES = {
    "pandora_params_default": [ctypes.POINTER(Params)],
    "pandora_strerror": [ctypes.c_int],
    "pandora_params_sizeof": [],
    "pandora_device_count": [ctypes.POINTER(ctypes.c_int)],
    "pandora_sizes": [ctypes.POINTER(Params), ctypes.POINTER(_i32), ctypes.POINTER(_i32), ctypes.POINTER(_i32),
                      ctypes.POINTER(_i64), ctypes.POINTER(_i32)],
    "pandora_create": [ctypes.POINTER(Params), ctypes.POINTER(_vp)],
    "pandora_destroy": [_vp],
    "pandora_set_stream": [_vp, _vp],
    "pandora_set_state": [_vp, _dp, _dp, _dp],
    "pandora_get_state": [_vp, _dp, _dp, _dp],
    "pandora_set_rk": [_vp, _dp, _dp, _dp],
    "pandora_get_rk": [_vp, _dp, _dp, _dp],
    "pandora_forcing_size": [_vp, ctypes.POINTER(_i64)],
    "pandora_set_forcing": [_vp, _dp, _dp, _dp],
    "pandora_get_forcing": [_vp, _dp, _dp, _dp],
    "pandora_state_device_ptrs": [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp)],
    "pandora_init_fluid": [_vp],
    "pandora_set_particles": [_vp, _i64, _dp, _dp, _dp, _dp, _dp],
    "pandora_get_particles": [_vp, _i64, _dp, _dp, _dp, _dp, _dp],
    "pandora_init_particles": [_vp],
    "pandora_rk3_step": [_vp, _i32, _dp, _dp],
    "pandora_rk3_advance": [_vp, _i32, _i32, _i32, _dp],
    "pandora_rk3_stage": [_vp, _i32, _i32, ctypes.c_double, _dp],
    "pandora_stats": [_vp, _dp, _i32, _dp, _dp, _dp],
    "pandora_last_step_stats": [_vp, _dp, _i32, _dp, _dp, _dp],
    "pandora_nonlinear": [_vp, _dp, _dp, _dp],
    "pandora_realspace_stats": [_vp, _dp, _i32],
    "pandora_x_correlation": [_vp, _dp, _i32],
    "pandora_particle_stats": [_vp, _dp, _i32],
    "pandora_get_physical_velocity": [_vp, _dp, _dp, _dp],
    "pandora_check_status": [_vp],
    "pandora_launches_per_step": [_vp, ctypes.POINTER(_i32)],
    "pandora_profile_pass": [_vp, _i32, _i32],
    "pandora_pass_bytes": [_vp, _i32, _dp],
    "pandora_set_pass_timing": [_vp, _i32],
    "pandora_pass_times": [_vp, ctypes.POINTER(ctypes.c_float)],
    "pandora_frame": [_vp, _dp, _dp],
    "pandora_nonlinear_static": [ctypes.POINTER(Params), _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "pandora_batch_bytes": [ctypes.POINTER(Params), _i32, ctypes.POINTER(_i64)],
    "pandora_batch_create": [ctypes.POINTER(Params), _i32, ctypes.POINTER(_vp)],
    "pandora_batch_destroy": [_vp],
    "pandora_batch_capacity": [_vp, ctypes.POINTER(_i32), ctypes.POINTER(_i32)],
    "pandora_batch_admit": [_vp, ctypes.POINTER(Params), ctypes.POINTER(_i32)],
    "pandora_batch_release": [_vp, _i32],
    "pandora_batch_step": [_vp, _i32, ctypes.POINTER(_i64)],
    "pandora_batch_finish": [_vp, _i32, ctypes.POINTER(_i64)],
    "pandora_batch_ticket_done": [_vp, _i64, ctypes.POINTER(_i32)],
    "pandora_batch_result_stats": [_vp, _i32, _dp, _i32, _dp, _dp],
    "pandora_batch_sync": [_vp],
    "pandora_batch_launches_per_step": [_vp, ctypes.POINTER(_i32)],
    "pandora_batch_member_time": [_vp, _i32, ctypes.POINTER(_i32), _dp, _dp],
    "pandora_batch_get_state": [_vp, _i32, _dp, _dp, _dp],
    "pandora_batch_get_particles": [_vp, _i32, _i64, _dp, _dp, _dp, _dp, _dp],
    "pandora_batch_last_step_stats": [_vp, _i32, _dp, _i32, _dp, _dp],
}
_RESTYPES = {"pandora_strerror": ctypes.c_char_p}


def lib_path() -> str:
    return LIB_PATH


def load(build_if_missing: bool = False):
    """Load the shared library (raises FileNotFoundError if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if build_if_missing:
            import importlib.util
            spec = importlib.util.spec_from_file_location("_pandora_build", os.path.join(PKG_ROOT, "build.py"))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            mod.build()
        else:
            raise FileNotFoundError(f"{LIB_PATH} not built; run python {os.path.join(PKG_ROOT, 'build.py')}")
    L = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    if L.pandora_params_sizeof() != ctypes.sizeof(Params):
        raise RuntimeError("pandora_params layout mismatch between Python and the library")
    _lib = L
    return L


def check(status: int, where: str) -> None:
    if status != OK:
        msg = load().pandora_strerror(status)
        raise PandoraError(status, where, msg.decode() if msg else "?")


def device_count() -> int:
    n = ctypes.c_int(0)
    st = load().pandora_device_count(ctypes.byref(n))
    return n.value if st == OK else 0
