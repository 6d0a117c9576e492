"""Batches of simulations of one class, stepped together (pandora_batch_*).

A batch has a fixed number of slots.  Admitting a member starts a fresh
simulation in a free slot (seeded field, step 1, time 0); every call of
``step(n)`` advances all occupied slots by n RK3 steps, each kernel launch serving
up to 32 members; a member's result is the same as that of the same parameters
run alone in a ``Simulation``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .params import Params



def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def class_key(p: Params) -> tuple:
    """The parameters that put two simulations in the same batch class."""
    npart = int(p.p_np_global) if p.p_track_part else 0
    return (p.nodes_x, p.nodes_y, p.nodes_z, p.precision, p.f_type, p.ns_deformed, p.b110, p.b220, p.b330,
            p.dealiasing, p.les_cutoff, p.rk3_viscous, npart, p.p_interp_order if npart else 0, float(p.force_kf))


def batch_bytes(p: Params, capacity: int) -> int:
    L = _lib.load()
    q = p.copy()
    b = ctypes.c_int64()
    _lib.check(L.pandora_batch_bytes(ctypes.byref(q), capacity, ctypes.byref(b)), "pandora_batch_bytes")
    return b.value


class Batch:
    def __init__(self, cls: Params, capacity: int):
        self.L = _lib.load()
        self.cls = cls.copy()
        self.capacity = capacity
        h = ctypes.c_void_p()
        _lib.check(self.L.pandora_batch_create(ctypes.byref(self.cls), capacity, ctypes.byref(h)),
                   "pandora_batch_create")
        self.h = h
        nki, nkj, nkk, kk = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        modes = ctypes.c_int64()
        _lib.check(self.L.pandora_sizes(ctypes.byref(self.cls), ctypes.byref(nki), ctypes.byref(nkj),
                                        ctypes.byref(nkk), ctypes.byref(modes), ctypes.byref(kk)), "pandora_sizes")
        self.shape = (nki.value, nkj.value, nkk.value)
        self.kkmax = kk.value
        self.np = int(self.cls.p_np_global) if self.cls.p_track_part else 0
        self.free = list(range(capacity))

    def close(self):
        if getattr(self, "h", None):
            self.L.pandora_batch_destroy(self.h)
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

    def admit(self, p: Params, slot: int | None = None) -> int:
        """Start a member (in `slot`, or the first free slot); returns the slot."""
        q = p.copy()
        s = ctypes.c_int32(-1 if slot is None else slot)
        _lib.check(self.L.pandora_batch_admit(self.h, ctypes.byref(q), ctypes.byref(s)), "pandora_batch_admit")
        if s.value in self.free:
            self.free.remove(s.value)
        return s.value

    def release(self, slot: int) -> None:
        _lib.check(self.L.pandora_batch_release(self.h, slot), "pandora_batch_release")
        self.free.append(slot)

    def step(self, n: int = 1) -> int:
        """Enqueue n steps of every member; returns a ticket (see ``done``)."""
        t = ctypes.c_int64()
        _lib.check(self.L.pandora_batch_step(self.h, n, ctypes.byref(t)), "pandora_batch_step")
        return t.value

    def finish(self, slot: int) -> int:
        """Free the slot, keeping its member's last-step statistics (``result_stats``
        once the returned ticket is done).  Does not wait."""
        t = ctypes.c_int64()
        _lib.check(self.L.pandora_batch_finish(self.h, slot, ctypes.byref(t)), "pandora_batch_finish")
        return t.value      # the slot rejoins ``free`` through ``reuse`` once its result is read

    def reuse(self, slot: int) -> None:
        self.free.append(slot)

    def done(self, ticket: int) -> bool:
        d = ctypes.c_int32()
        _lib.check(self.L.pandora_batch_ticket_done(self.h, ticket, ctypes.byref(d)), "pandora_batch_ticket_done")
        return bool(d.value)

    def result_stats(self, slot: int):
        ek = np.zeros(self.kkmax)
        tke, eps = ctypes.c_double(), ctypes.c_double()
        _lib.check(self.L.pandora_batch_result_stats(self.h, slot, _ptr(ek), self.kkmax, ctypes.byref(tke),
                                                     ctypes.byref(eps)), "pandora_batch_result_stats")
        return ek, tke.value, eps.value

    def sync(self) -> None:
        _lib.check(self.L.pandora_batch_sync(self.h), "pandora_batch_sync")

    def launches_per_step(self) -> int:
        n = ctypes.c_int32()
        _lib.check(self.L.pandora_batch_launches_per_step(self.h, ctypes.byref(n)), "pandora_batch_launches_per_step")
        return n.value

    def member_time(self, slot: int):
        """(next step number, time, dt) of the member in `slot`."""
        ts, t, dt = ctypes.c_int32(), ctypes.c_double(), ctypes.c_double()
        _lib.check(self.L.pandora_batch_member_time(self.h, slot, ctypes.byref(ts), ctypes.byref(t), ctypes.byref(dt)),
                   "pandora_batch_member_time")
        return ts.value, t.value, dt.value

    def get_state(self, slot: int):
        out = [np.zeros(self.shape, np.complex128) for _ in range(3)]
        _lib.check(self.L.pandora_batch_get_state(self.h, slot, *[_ptr(x.view(np.float64)) for x in out]),
                   "pandora_batch_get_state")
        return out

    def get_particles(self, slot: int):
        n = self.np
        xp, up, ur, pr = (np.zeros((n, 3)) for _ in range(4))
        dp = np.zeros(n)
        _lib.check(self.L.pandora_batch_get_particles(self.h, slot, n, _ptr(xp), _ptr(up), _ptr(ur), _ptr(pr),
                                                      _ptr(dp)), "pandora_batch_get_particles")
        return xp, up, ur, pr, dp

    def last_step_stats(self, slot: int):
        ek = np.zeros(self.kkmax)
        tke, eps = ctypes.c_double(), ctypes.c_double()
        _lib.check(self.L.pandora_batch_last_step_stats(self.h, slot, _ptr(ek), self.kkmax, ctypes.byref(tke),
                                                        ctypes.byref(eps)), "pandora_batch_last_step_stats")
        return ek, tke.value, eps.value
