"""ctypes front-end of the CPU oracle (liboracle.so built from pandora_oracle.c).

TEST INFRASTRUCTURE ONLY: the parity checker and the timed CPU baseline.  The
product never imports this module; only tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py do.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
_PKG = os.path.join(ROOT, "pandora-2.0_b200")
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)
from pandora.params import Params  # noqa: E402  (boundary struct layout)

LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    src = os.path.join(HERE, "pandora_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        vp, dp, i32, i64 = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_long
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [ctypes.POINTER(Params)]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_modes.restype = i64
        L.oracle_modes.argtypes = [vp]
        L.oracle_kkmax.restype = i32
        L.oracle_kkmax.argtypes = [vp]
        L.oracle_force_nk.restype = i32
        L.oracle_force_nk.argtypes = [vp]
        for n in ("oracle_set_state", "oracle_get_state", "oracle_set_rk", "oracle_get_rk",
                  "oracle_get_nl", "oracle_get_forcing", "oracle_get_physical", "oracle_nonlinear"):
            getattr(L, n).argtypes = [vp, dp, dp, dp]
        L.oracle_ucfl.restype = ctypes.c_double
        L.oracle_ucfl.argtypes = [vp]
        L.oracle_status.restype = i32
        L.oracle_status.argtypes = [vp]
        L.oracle_fft.restype = i32
        L.oracle_fft.argtypes = [i32, i32, dp, dp]
        L.oracle_set_particles.argtypes = [vp, i64, dp, dp, dp, dp, dp]
        L.oracle_get_particles.argtypes = [vp, dp, dp, dp, dp, dp]
        L.oracle_init_particles.argtypes = [vp]
        L.oracle_interpolate.argtypes = [vp, i64, dp, dp]
        L.oracle_stats.argtypes = [vp, dp, dp, dp]
        L.oracle_init_fluid.argtypes = [vp]
        L.oracle_init_taylor_green_reverse.argtypes = [vp]
        L.oracle_stage.restype = i32
        L.oracle_stage.argtypes = [vp, i32, i32, dp]
        L.oracle_step.restype = i32
        L.oracle_step.argtypes = [vp, i32, dp, dp]
        L.oracle_threads.restype = i32
        L.oracle_update_b.argtypes = [vp, i32, ctypes.c_double]
        L.oracle_get_b.argtypes = [vp, dp, dp]
        L.oracle_remesh_due.restype = i32
        L.oracle_remesh_due.argtypes = [vp, i32]
        L.oracle_force_calls_per_stage.restype = i64
        L.oracle_force_calls_per_stage.argtypes = [vp]
        L.oracle_realspace_sums.argtypes = [vp, dp]
        L.oracle_x_correlation.argtypes = [vp, dp]
        _lib = L
    return _lib


def _ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def fft(x: np.ndarray, sign: int) -> np.ndarray:
    """Unnormalised DFT of a complex line with the oracle's FFT (sign -1 forward)."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.complex128)).view(np.float64)
    out = np.zeros_like(a)
    assert lib().oracle_fft(len(x), sign, _ptr(a), _ptr(out)) == 0
    return out.view(np.complex128)


class Oracle:
    """One CPU simulation in the reference layout: u[c] is complex (NKI, NKJ, NKK)."""

    def __init__(self, p: Params):
        self.p = p.copy()
        self.L = lib()
        self.h = self.L.oracle_create(ctypes.byref(self.p))
        if not self.h:
            raise MemoryError("oracle_create failed")
        self.nki = p.nodes_x // 3 + 1
        self.nkj = 2 * (p.nodes_y // 3) + 1
        self.nkk = 2 * (p.nodes_z // 3) + 1
        self.shape = (self.nki, self.nkj, self.nkk)
        self.kkmax = self.L.oracle_kkmax(self.h)
        self.fnk = self.L.oracle_force_nk(self.h)

    def close(self):
        if self.h:
            self.L.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _three(self, fn, shape):
        a = [np.zeros(shape + (2,), np.float64) for _ in range(3)]
        fn(self.h, *[_ptr(x) for x in a])
        return [x.view(np.complex128)[..., 0] for x in a]

    def set_state(self, u):
        a = [np.ascontiguousarray(np.asarray(c, np.complex128)).view(np.float64) for c in u]
        self.L.oracle_set_state(self.h, *[_ptr(x) for x in a])

    def get_state(self):
        return self._three(self.L.oracle_get_state, self.shape)

    def set_rk(self, r):
        a = [np.ascontiguousarray(np.asarray(c, np.complex128)).view(np.float64) for c in r]
        self.L.oracle_set_rk(self.h, *[_ptr(x) for x in a])

    def get_rk(self):
        return self._three(self.L.oracle_get_rk, self.shape)

    def nonlinear(self):
        return self._three(self.L.oracle_nonlinear, self.shape)

    def realspace_sums(self):
        """f_FluidstatsRs2D's raw sums and maxima of the current state (25 values)."""
        out = np.zeros(25)
        self.L.oracle_realspace_sums(self.h, _ptr(out))
        return out

    def x_correlation(self):
        """TS_CORR's lag sums temp_r1i (NX/2 + 1 values) and lint11 (last), as the reference
        accumulates them."""
        out = np.zeros(self.p.nodes_x // 2 + 2)
        self.L.oracle_x_correlation(self.h, _ptr(out))
        return out

    def get_forcing(self):
        w = 2 * self.fnk + 1
        return self._three(self.L.oracle_get_forcing, (self.fnk + 1, w, w))

    def get_physical(self):
        p = self.p
        a = [np.zeros((p.nodes_z, p.nodes_y, p.nodes_x)) for _ in range(3)]
        self.L.oracle_get_physical(self.h, *[_ptr(x) for x in a])
        return a

    def init_fluid(self):
        self.L.oracle_init_fluid(self.h)

    def init_taylor_green_reverse(self):
        self.L.oracle_init_taylor_green_reverse(self.h)

    def set_particles(self, xp, up=None, uprk=None, prk=None, dp=None):
        n = len(xp)
        f = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
        self.L.oracle_set_particles(self.h, n, _ptr(f(xp)), _ptr(f(up)), _ptr(f(uprk)), _ptr(f(prk)),
                                    _ptr(f(dp)))

    def get_particles(self, n):
        xp, up, ur, pr = (np.zeros((n, 3)) for _ in range(4))
        dp = np.zeros(n)
        self.L.oracle_get_particles(self.h, _ptr(xp), _ptr(up), _ptr(ur), _ptr(pr), _ptr(dp))
        return xp, up, ur, pr, dp

    def init_particles(self):
        self.L.oracle_init_particles(self.h)

    def interpolate(self, xp):
        xp = np.ascontiguousarray(xp, np.float64)
        uf = np.zeros_like(xp)
        self.L.oracle_interpolate(self.h, len(xp), _ptr(xp), _ptr(uf))
        return uf

    def stats(self):
        ek = np.zeros(self.kkmax)
        tke, eps = ctypes.c_double(), ctypes.c_double()
        self.L.oracle_stats(self.h, _ptr(ek), ctypes.byref(tke), ctypes.byref(eps))
        return ek, tke.value, eps.value

    def ucfl(self):
        return self.L.oracle_ucfl(self.h)

    def status(self):
        return self.L.oracle_status(self.h)

    def stage(self, stage, tstep, dt):
        d = ctypes.c_double(dt)
        rc = self.L.oracle_stage(self.h, stage, tstep, ctypes.byref(d))
        if rc:
            raise RuntimeError(f"oracle_stage failed: {rc}")
        return d.value

    def step(self, tstep, simtime):
        t, d = ctypes.c_double(simtime), ctypes.c_double(0.0)
        rc = self.L.oracle_step(self.h, tstep, ctypes.byref(t), ctypes.byref(d))
        if rc:
            raise RuntimeError(f"oracle_step failed: {rc}")
        return t.value, d.value

    def frame(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        self.L.oracle_get_b(self.h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def update_b(self, tstep, simtime):
        self.L.oracle_update_b(self.h, tstep, simtime)

    def remesh_due(self, tstep):
        return bool(self.L.oracle_remesh_due(self.h, tstep))

    def force_calls_per_stage(self):
        return self.L.oracle_force_calls_per_stage(self.h)


def threads() -> int:
    return lib().oracle_threads()
