"""Deviation of a variant of the step from the FP64 explicit form of the same run: the
FP32-mixed form (default), or the integrating-factor viscous form (``--viscous``).

Both runs start from the same seeded field (the mixed form rounds the FP64 initial
field once), take the same steps on the same GPU, and are compared at the end:
relative L2 of u over all stored modes, relative L2 of E(k), and the relative error
of epsilon; both step times are reported.  The fields are compared on the device
(views of the state buffers through __cuda_array_interface__), so a 1024^3 state
never crosses to the host.

    python -m pandora.mixed_error --workload iso_forced --n 1024 --steps 200
    python -m pandora.mixed_error --workload iso_decay --n 64 --steps 100 --viscous
"""
from __future__ import annotations

import argparse
import json
import sys

import numpy as np

from .params import PREC_FP32_MIXED, PREC_FP64, VISCOUS_EXPLICIT, VISCOUS_INTEGRATING_FACTOR, Params, workload_params
from .rk3 import Simulation


class _DeviceArray:
    """A flat device buffer for torch.as_tensor (no copy)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def _state_views(sim: Simulation, mixed: bool):
    import ctypes
    import torch
    ptrs = [ctypes.c_void_p() for _ in range(3)]
    sim.L.pandora_state_device_ptrs(sim.h, *[ctypes.byref(q) for q in ptrs])
    n = 2 * int(np.prod(sim.shape))
    ts = "<f4" if mixed else "<f8"
    return [torch.as_tensor(_DeviceArray(q.value, n, ts), device="cuda") for q in ptrs]


def compare(p: Params, steps: int, viscous: bool = False) -> dict:
    """viscous=False: FP32-mixed against FP64 (explicit viscosity); True: FP64 with the
    integrating factor against FP64 explicit (the variant's figures keep the key names
    of the mixed form: fp32_mixed = the variant)."""
    import torch
    q64 = Params.from_buffer_copy(p)
    q64.precision = PREC_FP64
    q64.rk3_viscous = VISCOUS_EXPLICIT
    q32 = Params.from_buffer_copy(p)
    if viscous:
        q32.precision = PREC_FP64
        q32.rk3_viscous = VISCOUS_INTEGRATING_FACTOR
    else:
        q32.precision = PREC_FP32_MIXED
    out = {"grid": [p.nodes_x, p.nodes_y, p.nodes_z], "steps": steps,
           "variant": "integrating_factor" if viscous else "fp32_mixed"}
    sims = []
    for q in (q64, q32):
        s = Simulation(q)
        s.init_fluid()
        if q.p_track_part and q.p_np_global > 0:
            s.init_particles()
        sims.append(s)
    for name, s in (("fp64", sims[0]), ("fp32_mixed", sims[1])):
        s.advance(2, sync=True)                      # builds the step graph
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        s.advance(steps - 2, sync=True)
        e1.record()
        torch.cuda.synchronize()
        out[f"ms_per_step_{name}"] = e0.elapsed_time(e1) / max(steps - 2, 1)
    a, b = sims
    ua, ub = _state_views(a, False), _state_views(b, not viscous)
    num = sum(float(torch.sum((x - y.double()) ** 2)) for x, y in zip(ua, ub))
    den = sum(float(torch.sum(x ** 2)) for x in ua)
    out["rel_l2_u"] = (num / den) ** 0.5
    ek_a, _, eps_a, _ = a.stats()
    ek_b, _, eps_b, _ = b.stats()
    out["rel_l2_ek"] = float(np.linalg.norm(ek_b - ek_a) / np.linalg.norm(ek_a))
    out["rel_eps"] = float(abs(eps_b - eps_a) / abs(eps_a))
    out["speedup_fp32_mixed"] = out["ms_per_step_fp64"] / out["ms_per_step_fp32_mixed"]
    for s in sims:
        s.close()
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", default="iso_forced")
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--np", type=int, default=None, help="particles (workloads with tracers)")
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--viscous", action="store_true", help="the integrating-factor form against the explicit one")
    a = ap.parse_args(argv)
    p = workload_params(a.workload, a.n)
    if a.np is not None:
        p.p_np_global = a.np
        p.p_track_part = 1 if a.np > 0 else 0
    r = compare(p, a.steps, viscous=a.viscous)
    r["workload"] = a.workload
    print(json.dumps(r), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
