"""Namelist parameters of the RK3 step, mirrored as the C struct ``pandora_params``.

The fields are the ip_file.in namelist entries that the reference's RK3 path reads
(src/pg_control.f90:385-436, values of src/pg_parameters.f90).  ``Params`` is a
ctypes Structure with the exact layout of ``pandora_params`` in
include/pandora_gpu.h; ``read_namelist`` parses the subset of Fortran namelist
syntax that conf/ip_file.in uses.
"""
from __future__ import annotations

import ctypes
import math
import re

F_ISOTROPIC = 1
F_SHEAR_DNS = 2
F_ISOTROPIC_DEFORMED = 5
RK3_TIMESTEP_DECIDE = 1
RK3_TIMESTEP_FIXED = 2
RK3_TIMESTEP_CFL = 3
NS_BF_ROT = 1
NS_R_CONV = 2       # convective Rogallo form, 12 transformed fields (src/pf_rk3.f90:1717-1774)
NS_R_ROT = 3        # laboratory components on the sheared grid (src/pf_rk3.f90 R-rot)
F_INIT_NULL = 0
F_INIT_GAUSS = 3
F_INIT_KERR = 4
F_INIT_AHMED_ELGHOBASHI = 10
P_INIT_RANDOM = 2
PREC_FP64 = 0
PREC_FP32_MIXED = 1   # FP32 fields and transforms, FP64 bookkeeping (include/pandora_gpu.h)
VISCOUS_EXPLICIT = 0  # the reference's -F_NU k^2 u in every stage's right-hand side
VISCOUS_INTEGRATING_FACTOR = 1   # exp(-F_NU k^2 dc dt) factors per stage (include/pandora_gpu.h)


class Params(ctypes.Structure):
    """ctypes mirror of ``pandora_params`` (include/pandora_gpu.h)."""

    _fields_ = [
        ("nodes_x", ctypes.c_int32), ("nodes_y", ctypes.c_int32), ("nodes_z", ctypes.c_int32),
        ("b110", ctypes.c_int32), ("b220", ctypes.c_int32), ("b330", ctypes.c_int32),
        ("f_rho", ctypes.c_double), ("f_nu", ctypes.c_double),
        ("f_type", ctypes.c_int32),
        ("f_deform_s", ctypes.c_double),
        ("f_remesh_t", ctypes.c_int32),
        ("rk3_timestep", ctypes.c_int32),
        ("rk3_cfl", ctypes.c_double), ("rk3_dt", ctypes.c_double),
        ("ns_deformed", ctypes.c_int32),
        ("dealiasing", ctypes.c_int32),
        ("tsteps", ctypes.c_int32),
        ("f_init_type", ctypes.c_int32),
        ("f_init_u0", ctypes.c_double), ("f_init_kp", ctypes.c_double), ("f_init_kv", ctypes.c_double),
        ("f_init_kstart", ctypes.c_double), ("f_init_kend", ctypes.c_double),
        ("f_init_epsilon", ctypes.c_double),
        ("force_tf", ctypes.c_double), ("force_sigma", ctypes.c_double), ("force_kf", ctypes.c_double),
        ("force_stop", ctypes.c_int32),
        ("p_track_part", ctypes.c_int32),
        ("p_init_type", ctypes.c_int32),
        ("p_np_global", ctypes.c_int64),
        ("p_interp_order", ctypes.c_int32),
        ("p_ts_release", ctypes.c_int32),
        ("p_rho", ctypes.c_double),
        ("p_dia_vals", ctypes.c_double),
        ("seed_fluid", ctypes.c_uint64), ("seed_force", ctypes.c_uint64),
        ("seed_particles", ctypes.c_uint64),
        ("precision", ctypes.c_int32),
        ("rk3_viscous", ctypes.c_int32),
        ("les_cutoff", ctypes.c_double),
        ("x_lines_per_warp", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 3),
    ]

    def copy(self) -> "Params":
        q = Params()
        ctypes.memmove(ctypes.byref(q), ctypes.byref(self), ctypes.sizeof(Params))
        return q

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_ if not n.startswith("reserved")}


def default_params(n: int = 32) -> Params:
    """Defaults of conf/ip_file.in, with NODES = n and the isotropic flow type."""
    p = Params()
    p.nodes_x = p.nodes_y = p.nodes_z = n
    p.b110 = p.b220 = p.b330 = 1
    p.f_rho, p.f_nu = 1.0, 0.025
    p.f_type = F_ISOTROPIC
    p.f_deform_s, p.f_remesh_t = 28.3, 32
    p.rk3_timestep, p.rk3_cfl, p.rk3_dt = RK3_TIMESTEP_DECIDE, 0.75, 0.01
    p.ns_deformed, p.dealiasing, p.les_cutoff = NS_BF_ROT, 1, 1.0
    p.tsteps = 10
    p.f_init_type, p.f_init_u0, p.f_init_kp, p.f_init_kv = F_INIT_KERR, 0.1, 11.0, 20.0
    p.f_init_kstart, p.f_init_kend, p.f_init_epsilon = 5.0, 10.0, 0.0
    p.force_tf, p.force_sigma, p.force_kf, p.force_stop = 0.2, 0.03743, 2.829, 99999
    p.p_track_part, p.p_init_type, p.p_np_global = 0, P_INIT_RANDOM, 10
    p.p_interp_order, p.p_ts_release = 4, 1000
    p.p_rho, p.p_dia_vals = 1000.0, 0.01514314
    p.seed_fluid, p.seed_force, p.seed_particles = 1, 2, 3
    p.precision = PREC_FP64
    return p


def workload_params(name: str, n: int | None = None) -> Params:
    """The named synthetic workloads as reference parameters.

    ``iso_decay``: decaying isotropic turbulence, nu=0.01, dt=0.005 fixed, no
    forcing, Ahmed/Elghobashi spectrum with U0 = 2/3 u0^2 (u0=1, kp=4).
    ``iso_forced_particles``: forced isotropic turbulence, nu=0.002, dt=0.002
    fixed, OU forcing on |k| <= 2.5 with sigma^2 = P / (100 T_F) for an injected
    power P = 0.1 (the factor 100 is a calibration measured on this forcing, not
    the reference's e* = sigma^2 T_F), kp=3, 2^20 tracers
    (P_INIT_RANDOM, 4th-order interpolation, released at step 1).
    ``iso_forced``: the same forcing at nu=0.0008, dt=0.001, no particles (1024^3).
    ``shear``: homogeneous shear S=1 in the Rogallo frame (BF-rot), B110=2, 2^18 tracers.
    """
    if name == "iso_decay":
        p = default_params(n or 64)
        p.f_nu, p.rk3_timestep, p.rk3_dt, p.tsteps = 0.01, RK3_TIMESTEP_FIXED, 0.005, 100
        p.force_stop = 0
        p.f_init_type, p.f_init_kp, p.f_init_u0 = F_INIT_AHMED_ELGHOBASHI, 4.0, 2.0 / 3.0
        p.p_track_part = 0
        return p
    if name == "iso_forced_particles":
        p = default_params(n or 256)
        p.f_nu, p.rk3_timestep, p.rk3_dt, p.tsteps = 0.002, RK3_TIMESTEP_FIXED, 0.002, 500
        p.force_kf, p.force_tf, p.force_stop = 2.5, 0.2, 100000
        # injected power P = 0.1.  The reference prints e* = sigma^2 T_F
        # (src/pf_force.f90:394-424) as its forcing's power, which does not count
        # the ~80 forced modes; the injection measured on this forcing (the mean
        # of sum_k Re(f . conj u) over many steps) is P ~ 100 sigma^2 T_F, an
        # observed calibration, so sigma^2 = P / (100 T_F)
        p.force_sigma = math.sqrt(0.1 / (100.0 * 0.2))
        p.f_init_type, p.f_init_kp, p.f_init_u0 = F_INIT_AHMED_ELGHOBASHI, 3.0, 2.0 / 3.0
        p.p_track_part, p.p_init_type, p.p_np_global = 1, P_INIT_RANDOM, 1 << 20
        p.p_interp_order, p.p_ts_release, p.p_dia_vals = 4, 1, 0.0
        return p
    if name == "iso_forced":
        # forced isotropic turbulence without particles at the mixed-precision size:
        # nu = 0.0008, dt = 0.001, forcing as iso_forced_particles, kp = 3
        p = workload_params("iso_forced_particles", n or 1024)
        p.f_nu, p.rk3_dt, p.tsteps = 0.0008, 0.001, 200
        p.p_track_part, p.p_np_global = 0, 0
        return p
    if name == "shear":
        # homogeneous shear dU1/dx3 = S in Rogallo (moving-frame) coordinates,
        # BF-rot formulation, lab box 4pi x 2pi x 2pi (B110 = 2), fixed dt =
        # (0.5/S)/F_REMESH_T, remesh every S t = B110 (src/pf_rk3.f90:3921-4026)
        p = default_params(n or 512)
        p.b110 = 2
        p.f_type, p.ns_deformed, p.f_deform_s = F_SHEAR_DNS, NS_BF_ROT, 1.0
        p.rk3_timestep, p.f_remesh_t, p.tsteps = RK3_TIMESTEP_DECIDE, 250, 3000
        p.f_nu, p.force_stop = 0.005, 0
        p.f_init_type, p.f_init_kp, p.f_init_u0 = F_INIT_AHMED_ELGHOBASHI, 4.0, (2.0 / 3.0) * 0.5 ** 2
        p.p_track_part, p.p_init_type, p.p_np_global = 1, P_INIT_RANDOM, 1 << 18
        p.p_interp_order, p.p_ts_release, p.p_dia_vals = 4, 1, 0.0
        return p
    raise ValueError(f"unknown workload {name!r}")


_NL_KEYS = {k.upper(): k for k, _ in Params._fields_}


def read_namelist(text: str, base: Params | None = None) -> Params:
    """Parse ``&nl_* key = value ... /`` groups (comments after ``!``) into Params.

    Keys that are not fields of Params are ignored, as the reference ignores keys
    that the RK3 path does not read.  ``RANDOM_SEED_FLUID`` / ``..._PARTICLES`` lists
    are folded into one 64-bit seed each.
    """
    p = base.copy() if base is not None else default_params()
    body = "\n".join(line.split("!", 1)[0] for line in text.splitlines())
    for group in re.findall(r"&\w+(.*?)/", body, flags=re.S):
        for key, val in re.findall(r"(\w+)\s*=\s*([^=\n]+?)(?=\s+\w+\s*=|\s*$)", group, flags=re.S | re.M):
            key = key.upper()
            vals = [v.strip() for v in val.replace("\n", " ").split(",") if v.strip()]
            if key in ("RANDOM_SEED_FLUID", "RANDOM_SEED_PARTICLES"):
                seed = 0
                for v in vals:
                    seed = (seed * 1000003 + int(float(v))) & ((1 << 64) - 1)
                setattr(p, "seed_fluid" if key.endswith("FLUID") else "seed_particles", seed)
                continue
            if key == "NODES_X":
                p.nodes_x = int(float(vals[0]))
                continue
            name = _NL_KEYS.get(key)
            if name is None or not vals:
                continue
            ctype = dict(Params._fields_)[name]
            v = vals[0].strip("'\"")
            if ctype in (ctypes.c_double,):
                setattr(p, name, float(v.replace("d", "e").replace("D", "e")))
            else:
                setattr(p, name, int(float(v)))
    return p
