"""Host-side mirror of the reference's RK3 interface, driving the CUDA library.

The reference keeps its fields module-global and exposes Fortran subroutines
(src/pg_rk3.f90:82 g_RK3Calc, src/pf_rk3.f90:40,121,161 f_RK3Stage1..3,
src/pp_control.f90:589 p_ControlInitialiseParticles, src/pf_fluidstats.f90:1293
f_FluidstatsFs, src/pf_initialise.f90 f_InitialiseInit).  ``Simulation`` owns
one device handle; the module-level functions with the reference's names act on
a current simulation set by ``ProgramInit``, the way the Fortran modules act on
their module state.  Errors that the reference turns into ``MPI_Abort`` or a
non-zero ``ierr`` raise ``PandoraError`` here.

Arrays use the reference layout: complex128 of shape (NKI, NKJ, NKK) per
component, NKI = NX/3+1, NKJ = 2(NY/3)+1, NKK = 2(NZ/3)+1.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .params import Params


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _as_f64(a, shape=None) -> np.ndarray:
    a = np.ascontiguousarray(a)
    if np.iscomplexobj(a):
        a = np.ascontiguousarray(a.astype(np.complex128, copy=False)).view(np.float64)
    else:
        a = np.ascontiguousarray(a, dtype=np.float64)
    return a


def realspace_normalise(raw, p) -> dict:
    """f_FluidstatsRsCollect's normalisation (src/pf_fluidstats.f90:960-1100) of the raw
    sums [u1u1 u2u2 u3u3 u1u2 u1u3 u2u3, u^3 (3), u^4 (3), w^2 (3), w^3 (3), w^4 (3),
    umax, wmax (3)]."""
    npts = float(p.nodes_x) * float(p.nodes_y) * float(p.nodes_z)
    r = {}
    for a, k in enumerate(("u1u1", "u2u2", "u3u3", "u1u2", "u1u3", "u2u3")):
        r[k] = raw[a] / npts
    for c in range(3):
        uu = r[("u1u1", "u2u2", "u3u3")[c]]
        r[f"skew{c + 1}"] = raw[6 + c] / npts / uu ** 1.5
        r[f"flat{c + 1}"] = raw[9 + c] / npts / uu ** 2
    rms = [raw[12], raw[13] / npts, raw[14] / npts]   # rmsvort1 unnormalised, as the reference
    rms = [x ** 0.5 for x in rms]
    for c in range(3):
        r[f"rmsvort{c + 1}"] = rms[c]
        r[f"skewvort{c + 1}"] = raw[15 + c] / npts / rms[c] ** 3
        r[f"flatvort{c + 1}"] = raw[18 + c] / npts / rms[c] ** 4
    r["ucfl"] = raw[21]
    for c in range(3):
        r[f"omegamax{c + 1}"] = raw[22 + c]
    r["lint11"] = 0.0   # without the correlation (TS_CORR > TSTEPS), src/pf_fluidstats.f90:1104-1105
    return r


def correlation_normalise(rsum, u1u1, p) -> dict:
    """f_FluidstatsRsCollect's finish of TS_CORR (src/pf_fluidstats.f90:1092-1105): r1i =
    temp_r1i / (rs_u1u1 N^3) at the lags l dx_laboratoryframe, l = 0..NX/2, and rs_lint11 =
    sum_l temp_r1i(l) dx_laboratoryframe / (rs_u1u1 N^3); ``u1u1`` is the normalised rs_u1u1."""
    npts = float(p.nodes_x) * float(p.nodes_y) * float(p.nodes_z)
    dxl = 2.0 * np.pi * float(p.b110) / float(p.nodes_x)
    rsum = np.asarray(rsum, dtype=np.float64)
    return {"r": np.arange(rsum.size) * dxl, "r1i": rsum / (u1u1 * npts),
            "lint11": float(np.sum(rsum * dxl)) / (u1u1 * npts)}


class Simulation:
    """One resident simulation on the current CUDA device."""

    def __init__(self, params: Params):
        self.L = _lib.load()
        self.p = params.copy()
        h = ctypes.c_void_p()
        _lib.check(self.L.pandora_create(ctypes.byref(self.p), ctypes.byref(h)), "pandora_create")
        self.h = h
        nki, nkj, nkk, kk = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        modes = ctypes.c_int64()
        _lib.check(self.L.pandora_sizes(ctypes.byref(self.p), ctypes.byref(nki), ctypes.byref(nkj),
                                        ctypes.byref(nkk), ctypes.byref(modes), ctypes.byref(kk)), "pandora_sizes")
        self.shape = (nki.value, nkj.value, nkk.value)
        self.modes = modes.value
        self.kkmax = kk.value
        nf = ctypes.c_int64()
        _lib.check(self.L.pandora_forcing_size(self.h, ctypes.byref(nf)), "pandora_forcing_size")
        nk = int(self.p.force_kf)
        self.force_shape = (nk + 1, 2 * nk + 1, 2 * nk + 1)
        self.np = int(self.p.p_np_global) if self.p.p_track_part else 0
        self.simtime = 0.0
        self.tstep = 0

    # ---- lifetime ----
    def close(self):
        if getattr(self, "h", None):
            self.L.pandora_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle: int | None):
        _lib.check(self.L.pandora_set_stream(self.h, ctypes.c_void_p(stream_handle or 0)), "pandora_set_stream")

    # ---- state ----
    def _put3(self, fn, arrs, name):
        a = [_as_f64(x) for x in arrs]
        _lib.check(fn(self.h, *[_dp(x) for x in a]), name)

    def _get3(self, fn, shape, name):
        out = [np.zeros(shape, np.complex128) for _ in range(3)]
        _lib.check(fn(self.h, *[_dp(x.view(np.float64)) for x in out]), name)
        return out

    def set_state(self, u):
        for c in u:
            if np.shape(c) != self.shape:
                raise ValueError(f"state component shape {np.shape(c)} != {self.shape}")
        self._put3(self.L.pandora_set_state, u, "pandora_set_state")

    def get_state(self):
        return self._get3(self.L.pandora_get_state, self.shape, "pandora_get_state")

    def set_rk(self, r):
        self._put3(self.L.pandora_set_rk, r, "pandora_set_rk")

    def get_rk(self):
        return self._get3(self.L.pandora_get_rk, self.shape, "pandora_get_rk")

    def set_forcing(self, f):
        self._put3(self.L.pandora_set_forcing, f, "pandora_set_forcing")

    def get_forcing(self):
        return self._get3(self.L.pandora_get_forcing, self.force_shape, "pandora_get_forcing")

    def init_fluid(self):
        _lib.check(self.L.pandora_init_fluid(self.h), "pandora_init_fluid")

    # ---- particles ----
    def init_particles(self):
        _lib.check(self.L.pandora_init_particles(self.h), "pandora_init_particles")

    def set_particles(self, xp, up=None, up_rk3=None, rk3=None, dp=None):
        n = len(xp)
        held = [None if a is None else _as_f64(a) for a in (xp, up, up_rk3, rk3, dp)]
        ptrs = [None if a is None else _dp(a) for a in held]
        _lib.check(self.L.pandora_set_particles(self.h, n, *ptrs), "pandora_set_particles")

    def get_particles(self):
        n = self.np
        xp, up, ur, pr = (np.zeros((n, 3)) for _ in range(4))
        dp = np.zeros(n)
        _lib.check(self.L.pandora_get_particles(self.h, n, _dp(xp), _dp(up), _dp(ur), _dp(pr), _dp(dp)),
                   "pandora_get_particles")
        return xp, up, ur, pr, dp

    # ---- restart files (PETSc binary, g_RestartPetscFluid / g_RestartPetscParticle) ----
    def write_restart(self, path: str, particle_path: str | None = None) -> None:
        from . import restart
        restart.write_fluid(path, self.get_state())
        if particle_path is not None:
            xp, up, _, _, dp = self.get_particles()
            restart.write_particles(particle_path, xp.T, up.T, dp)

    def read_restart(self, path: str, particle_path: str | None = None, scale: int = 1) -> None:
        """State (and particles) from restart files; `scale` = F_RESTART_SCALE: the
        file holds the field of a grid `scale` times coarser in every direction."""
        from . import restart
        if scale == 1:
            u = restart.read_fluid(path, self.shape)
        else:
            p = self.p
            ki, kj, kk = (p.nodes_x // scale) // 3, (p.nodes_y // scale) // 3, (p.nodes_z // scale) // 3
            u = restart.scale_fluid(restart.read_fluid(path, (ki + 1, 2 * kj + 1, 2 * kk + 1)), self.shape)
        self.set_state(u)
        if particle_path is not None:
            d = restart.read_particles(particle_path)
            xp = np.stack([d["xp1"], d["xp2"], d["xp3"]], axis=1)
            up = np.stack([d["up1"], d["up2"], d["up3"]], axis=1)
            self.set_particles(xp, up=up, dp=d["dp"])

    # ---- stepping ----
    def step(self, tstep: int | None = None) -> float:
        """g_RK3Calc: one RK3 step; returns dt."""
        if tstep is None:
            tstep = self.tstep + 1
        t = ctypes.c_double(self.simtime)
        d = ctypes.c_double(0.0)
        _lib.check(self.L.pandora_rk3_step(self.h, tstep, ctypes.byref(t), ctypes.byref(d)), "pandora_rk3_step")
        self.simtime, self.tstep = t.value, tstep
        return d.value

    def advance(self, nsteps: int, sync: bool = True) -> None:
        t = ctypes.c_double(self.simtime)
        _lib.check(self.L.pandora_rk3_advance(self.h, self.tstep + 1, nsteps, 1 if sync else 0, ctypes.byref(t)),
                   "pandora_rk3_advance")
        self.tstep += nsteps
        if sync:
            self.simtime = t.value

    def stage(self, stage: int, tstep: int, time: float, dt: float) -> float:
        d = ctypes.c_double(dt)
        _lib.check(self.L.pandora_rk3_stage(self.h, stage, tstep, time, ctypes.byref(d)), "pandora_rk3_stage")
        return d.value

    # ---- diagnostics ----
    def stats(self, last_step: bool = False):
        ek = np.zeros(self.kkmax)
        tke, eps, ucfl = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        fn = self.L.pandora_last_step_stats if last_step else self.L.pandora_stats
        _lib.check(fn(self.h, _dp(ek), self.kkmax, ctypes.byref(tke), ctypes.byref(eps), ctypes.byref(ucfl)),
                   "pandora_stats")
        return ek, tke.value, eps.value, ucfl.value

    def realspace_sums(self) -> np.ndarray:
        """Raw sums and maxima of `pandora_realspace_stats` (25 values)."""
        out = np.zeros(25)
        _lib.check(self.L.pandora_realspace_stats(self.h, _dp(out), 25), "pandora_realspace_stats")
        return out

    def realspace_stats(self, corr: bool = False) -> dict:
        """f_FluidstatsRs2D + f_FluidstatsRsCollect (src/pf_fluidstats.f90:827-1100) of the
        current state, normalised as the reference does (its rmsvort1 is not divided
        by the number of points, src/pf_fluidstats.f90:1057; that is kept).  With
        ``corr`` (a TS_CORR step) also the longitudinal autocorrelation ``r1i`` at the lags
        ``r`` and the integral length ``lint11``."""
        r = realspace_normalise(self.realspace_sums(), self.p)
        if corr:
            r.update(correlation_normalise(self.x_correlation_sums(), r["u1u1"], self.p))
        return r

    def x_correlation_sums(self) -> np.ndarray:
        """Raw lag sums of `pandora_x_correlation` (NX/2 + 1 values)."""
        out = np.zeros(self.p.nodes_x // 2 + 1)
        _lib.check(self.L.pandora_x_correlation(self.h, _dp(out), out.size), "pandora_x_correlation")
        return out

    def particle_stats(self) -> dict:
        """p_StatsPrimary (src/pp_stats.f90:119-200): particle velocity moments / NP and
        the mean particle kinetic energy."""
        out = np.zeros(7)
        _lib.check(self.L.pandora_particle_stats(self.h, _dp(out), 7), "pandora_particle_stats")
        n = float(self.p.p_np_global)
        names = ("u1u1", "u2u2", "u3u3", "u1u2", "u1u3", "u2u3")
        d = {k: out[a] / n for a, k in enumerate(names)}
        d["tke"] = 0.5 * (d["u1u1"] + d["u2u2"] + d["u3u3"])
        d["pken"] = out[6] / n
        return d

    def nonlinear(self):
        return self._get3(self.L.pandora_nonlinear, self.shape, "pandora_nonlinear")

    def device_state_ptrs(self):
        """Device addresses of u1..u3 (zero-copy): S complex values each, double2 in the
        FP64 form and float2 in the FP32-mixed form, valid until ``close``."""
        a, b, c = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        _lib.check(self.L.pandora_state_device_ptrs(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
                   "pandora_state_device_ptrs")
        return a.value, b.value, c.value

    def physical_velocity(self):
        p = self.p
        out = [np.zeros((p.nodes_z, p.nodes_y, p.nodes_x)) for _ in range(3)]
        _lib.check(self.L.pandora_get_physical_velocity(self.h, *[_dp(x) for x in out]),
                   "pandora_get_physical_velocity")
        return out

    def frame(self):
        """(bmat(1,3), binv(1,3)) of the moving frame (shear flow)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        _lib.check(self.L.pandora_frame(self.h, ctypes.byref(a), ctypes.byref(b)), "pandora_frame")
        return a.value, b.value

    def check_status(self) -> None:
        _lib.check(self.L.pandora_check_status(self.h), "pandora_check_status")

    def profile_pass(self, pass_id: int, reps: int) -> None:
        _lib.check(self.L.pandora_profile_pass(self.h, pass_id, reps), "pandora_profile_pass")

    def pass_bytes(self, pass_id: int) -> float:
        b = ctypes.c_double()
        _lib.check(self.L.pandora_pass_bytes(self.h, pass_id, ctypes.byref(b)), "pandora_pass_bytes")
        return b.value

    def set_pass_timing(self, passes: int) -> None:
        """Record a CUDA event pair around the passes in the bitmask (bit p-1 = pass p,
        0x3F = all six, 0 = off) in every stage of each step."""
        _lib.check(self.L.pandora_set_pass_timing(self.h, int(passes)), "pandora_set_pass_timing")

    def pass_times(self) -> np.ndarray:
        """Durations (ms) of the passes of the most recent step, [stage 1..3][pass 1..6]; -1 = not run."""
        out = (ctypes.c_float * 18)()
        _lib.check(self.L.pandora_pass_times(self.h, out), "pandora_pass_times")
        return np.array(out, dtype=np.float64).reshape(3, 6)

    def launches_per_step(self) -> int:
        n = ctypes.c_int32()
        _lib.check(self.L.pandora_launches_per_step(self.h, ctypes.byref(n)), "pandora_launches_per_step")
        return n.value


# ---------------------------------------------------------------------------
# reference-named entry points over a current simulation
# ---------------------------------------------------------------------------
_current: Simulation | None = None


def ProgramInit(params: Params) -> Simulation:
    """ProgramInit (src/pg_control.f90:52-146): allocate the resident state and
    initialise the fluid (and particles) from the seeds."""
    global _current
    if _current is not None:
        _current.close()
    sim = Simulation(params)
    f_InitialiseInit(sim)
    if params.p_track_part:
        sim.init_particles()
    _current = sim
    return sim


def _sim(sim: Simulation | None) -> Simulation:
    s = sim or _current
    if s is None:
        raise RuntimeError("no current simulation; call ProgramInit first")
    return s


def f_InitialiseInit(sim: Simulation | None = None) -> None:
    """f_InitialiseInit: seeded solenoidal field (src/pf_initialise.f90:97-512)."""
    _sim(sim).init_fluid()


def g_RK3Calc(tstep: int, simtime: float, sim: Simulation | None = None) -> float:
    """g_RK3Calc (src/pg_rk3.f90:82-129): returns the new simtime."""
    s = _sim(sim)
    s.simtime = simtime
    s.step(tstep)
    return s.simtime


def f_RK3Stage1(tstep: int, time: float, dt: float, sim: Simulation | None = None) -> float:
    return _sim(sim).stage(1, tstep, time, dt)


def f_RK3Stage2(tstep: int, time: float, dt: float, sim: Simulation | None = None) -> float:
    return _sim(sim).stage(2, tstep, time, dt)


def f_RK3Stage3(tstep: int, time: float, dt: float, sim: Simulation | None = None) -> float:
    return _sim(sim).stage(3, tstep, time, dt)


def f_FluidstatsFs(sim: Simulation | None = None):
    """Primary spectral statistics (src/pf_fluidstats.f90:1423-1576): E(k), tke, eps, ucfl."""
    return _sim(sim).stats()


def p_ControlInitialiseParticles(sim: Simulation | None = None) -> None:
    """P_INIT_RANDOM particle positions (src/pp_control.f90:663-707)."""
    _sim(sim).init_particles()
