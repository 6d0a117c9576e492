"""Ensemble server: independent simulations of uneven size, served as they arrive.

Requests (grid 32^3 to 256^3, isotropic or sheared, with or without tracers, FP64
or FP32-mixed) arrive over time.  Each belongs to a batch class (same grid,
precision, flow type, particle count); a class has one ``Batch`` whose slots are
the only device memory it uses, created when the class first appears and
admitted against an HBM budget (idle batches are evicted when another class needs
the room).  The loop is continuous batching: an arriving request takes a free
slot of its class at once, even while the other members are mid-run; every batch
with occupied slots is advanced a few steps at a time on its own stream, so the
classes' work overlaps on the GPU; a member that reaches its step count is read
out and its slot freed for the next request.  Batch schedules come from an
autotuner that measures member-steps/s per (grid, precision) at several capacities
(members per launch) and, for lines of up to 64 points, x-pass schedules (1, 2 or 4
lines per warp), and keeps the best pair.

    python -m pandora.ensemble --requests 2000 --load 0.8 --budget-gb 150
"""
from __future__ import annotations

import argparse
import collections
import json
import math
import os
import sys
import time
from dataclasses import dataclass, field

import numpy as np

from .batch import Batch, batch_bytes, class_key
from .params import PREC_FP32_MIXED, PREC_FP64, Params, workload_params
from .rk3 import Simulation

SIZES = (32, 48, 64, 96, 128, 192, 256)


@dataclass
class Request:
    rid: int
    params: Params
    steps: int
    arrival: float                 # seconds from the start of the trace
    variant: str
    admitted: float | None = None
    done: float | None = None
    result: dict = field(default_factory=dict)
    key: tuple | None = None       # class_key(params), computed once by the server

    @property
    def points(self) -> int:
        return self.params.nodes_x * self.params.nodes_y * self.params.nodes_z


def request_params(n: int, shear: bool, particles: int, precision: int, seed: int) -> Params:
    """One request of the ensemble trace as reference parameters: decaying isotropic
    turbulence (the 64^3 configuration's spectrum, nu = 0.01 * 64 / N) or homogeneous
    shear S = 1 with B110 = 1; `particles` tracers of order 4."""
    if shear:
        p = workload_params("shear", n)
        p.b110 = 1
        p.f_nu = 0.01 * 64.0 / n
    else:
        p = workload_params("iso_decay", n)
        p.f_nu = 0.01 * 64.0 / n
    p.p_track_part = 1 if particles > 0 else 0
    p.p_np_global = particles
    p.p_init_type, p.p_interp_order, p.p_ts_release, p.p_dia_vals = 2, 4, 1, 0.0
    p.precision = precision
    p.seed_fluid, p.seed_force, p.seed_particles = seed, 100000 + seed, 200000 + seed
    return p


def make_trace(n_requests: int, seed: int = 7, rate: float | None = None, steps: int = 200,
               variants=("fp64", "fp32_mixed"), particles: int = 1 << 14, sizes=SIZES) -> list[Request]:
    """The ensemble trace: N drawn with weight 1/N^2, 70% isotropic / 30% shear, 0 or
    `particles` tracers with equal probability, each request in every variant.
    Arrivals are Poisson at `rate` requests per second (None: all at time 0)."""
    rng = np.random.default_rng(seed)
    w = np.array([1.0 / (n * n) for n in sizes])
    w /= w.sum()
    out, t = [], 0.0
    for r in range(n_requests):
        if rate:
            t += rng.exponential(1.0 / rate)
        n = int(rng.choice(sizes, p=w))
        shear = rng.random() < 0.3
        npart = particles if rng.random() < 0.5 else 0
        for v in variants:
            prec = PREC_FP32_MIXED if v == "fp32_mixed" else PREC_FP64
            p = request_params(n, shear, npart, prec, seed=1 + r)
            out.append(Request(len(out), p, steps, t, v))
    return out


# ---------------------------------------------------------------------------
# capacity autotuner
# ---------------------------------------------------------------------------
def pick_capacity(rates: dict) -> int:
    """The smallest capacity whose member-steps/s is within 5% of the best measured one:
    a larger batch of a class reserves more memory and runs its free slots' CTAs while the
    trace leaves them empty, for a gain below the measurements' noise."""
    top = max(rates.values())
    return min(int(c) for c, r in rates.items() if r >= 0.95 * top)


def tune_capacity(n: int, precision: int, caps=(1, 2, 4, 8, 16, 32, 64), steps: int = 6,
                  max_bytes: int = 40 << 30) -> dict:
    """The batch schedule of a class: member-steps/s of a full batch of decaying-isotropic
    members at each capacity, for each x-pass schedule the length has (x lines per warp
    1, 2, 4 up to 64 points); the schedule with the highest rate, and at it the capacity
    of pick_capacity.  Returns {"best": cap, "xlpw": lines per warp, "rates": {cap:
    member-steps/s at that schedule}, "rates_by_xlpw": {...}}."""
    import torch
    lpws = (1, 2, 4) if n <= 64 else (1,)
    by_lpw = {}
    for lpw in lpws:
        rates = {}
        top = 0.0
        for cap in caps:
            p = request_params(n, False, 0, precision, seed=1)
            p.x_lines_per_warp = lpw
            if batch_bytes(p, cap) > max_bytes:
                break
            with Batch(p, cap) as b:
                for k in range(cap):
                    q = request_params(n, False, 0, precision, seed=1 + k)
                    q.x_lines_per_warp = lpw
                    b.admit(q)
                b.step(2)
                b.sync()
                t0 = time.perf_counter()
                b.step(steps)
                b.sync()
                rate = cap * steps / (time.perf_counter() - t0)
            rates[cap] = rate
            if rate < top:
                break
            top = max(top, rate)
        by_lpw[lpw] = rates
    torch.cuda.synchronize()
    best_lpw = max(by_lpw, key=lambda l: max(by_lpw[l].values()))
    return {"best": pick_capacity(by_lpw[best_lpw]), "xlpw": best_lpw, "rates": by_lpw[best_lpw],
            "rates_by_xlpw": by_lpw}


# Capacities measured on a B200 by tune_capacity (the starting table of autotune).
MEASURED_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotune_b200.json")


def autotune(sizes=SIZES, precisions=(PREC_FP64, PREC_FP32_MIXED), cache: str | None = None,
             start: str | None = MEASURED_TABLE) -> dict:
    """Batch capacity per (N, precision): from `cache` (JSON) if it exists, else from
    the measured table `start`; classes missing from both are measured now, and the
    table is written to `cache` when given."""
    table = {}
    src = cache if (cache and os.path.exists(cache)) else start
    if src and os.path.exists(src):
        with open(src) as fh:
            table = json.load(fh)
        for entry in table.values():   # the schedule and capacity follow from the stored rates
            by = entry.get("rates_by_xlpw")
            if by:
                lpw = max(by, key=lambda l: max(by[l].values()))
                entry["xlpw"], entry["rates"] = int(lpw), by[lpw]
            if entry.get("rates"):
                entry["best"] = pick_capacity(entry["rates"])
    changed = False
    for n in sizes:
        for prec in precisions:
            key = f"{n}/{prec}"
            if key not in table:
                table[key] = tune_capacity(n, prec)
                changed = True
    if cache and changed:
        with open(cache, "w") as fh:
            json.dump(table, fh, indent=1)
    return table


# ---------------------------------------------------------------------------
# the server loop
# ---------------------------------------------------------------------------
class Server:
    """The request loop.  Never waits on the GPU except to read a finished member's
    state when ``keep_state`` asks for it (tests): steps, finishes and admissions are
    enqueued on the batches' streams, completions are found by polling tickets."""

    def __init__(self, budget_bytes: int, capacity: dict, chunk: int = 8, inflight: int = 2,
                 keep_state: bool = False):
        self.budget = budget_bytes
        self.capacity = capacity          # "N/precision" -> {"best": capacity}
        self.chunk = chunk
        self.inflight = inflight
        self.keep_state = keep_state
        self.batches: dict[tuple, Batch] = {}
        self.bytes: dict[tuple, int] = {}
        self.members: dict[tuple, dict[int, list]] = collections.defaultdict(dict)   # key -> slot -> [req, left]
        self.tickets: dict[tuple, collections.deque] = collections.defaultdict(collections.deque)
        self.finishing: list = []         # (key, slot, ticket, request)
        self.peak_bytes = 0

    def _cap(self, p: Params) -> int:
        return int(self.capacity.get(f"{p.nodes_x}/{p.precision}", {"best": 1}).get("best", 1))

    def _xlpw(self, p: Params) -> int:
        """The class's x-pass schedule from the autotuner (0: the library's choice)."""
        return int(self.capacity.get(f"{p.nodes_x}/{p.precision}", {}).get("xlpw", 0))

    def _busy(self, key) -> bool:
        return bool(self.members[key]) or any(f[0] == key for f in self.finishing)

    def _batch_for(self, req: Request) -> Batch | None:
        key = req.key
        b = self.batches.get(key)
        if b is not None:
            return b
        cap = self._cap(req.params)
        need = batch_bytes(req.params, cap)
        while sum(self.bytes.values()) + need > self.budget:
            idle = [k for k in self.batches if not self._busy(k)]
            if not idle:
                return None
            k = idle[0]
            self.batches.pop(k).close()
            self.bytes.pop(k)
            self.tickets.pop(k, None)
        cls = req.params.copy()
        cls.x_lines_per_warp = self._xlpw(req.params)
        b = Batch(cls, cap)
        self.batches[key] = b
        self.bytes[key] = need
        self.peak_bytes = max(self.peak_bytes, sum(self.bytes.values()))
        return b

    def run(self, requests: list[Request], realtime: bool = True) -> dict:
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        # waiting requests, one arrival-ordered queue per class: an admission pass looks at
        # each class with waiting requests once (the classes in the order of their oldest
        # waiting request), not at every waiting request
        waiting: dict[tuple, collections.deque] = {}
        t0 = time.perf_counter()
        left = len(requests)
        while left:
            now = time.perf_counter() - t0
            while pending and (not realtime or pending[0].arrival <= now):
                r = pending.popleft()
                if r.key is None:
                    r.key = class_key(r.params)
                waiting.setdefault(r.key, collections.deque()).append(r)
            # admission: waiting requests of classes with a free slot
            for key in sorted(waiting, key=lambda k: waiting[k][0].arrival):
                q = waiting[key]
                b = self._batch_for(q[0])
                if b is None:
                    continue
                while q and b.free:
                    r = q.popleft()
                    slot = b.admit(r.params, b.free[0])   # the schedule is the batch's (results do not depend on it)
                    r.admitted = time.perf_counter() - t0
                    self.members[key][slot] = [r, r.steps]
                if not q:
                    del waiting[key]
            # keep `inflight` step chunks queued per batch; a member's finish follows
            # the chunk that completes it in stream order
            progressed = False
            for key, mem in self.members.items():
                if not mem:
                    continue
                b = self.batches[key]
                q = self.tickets[key]
                while q and b.done(q[0]):
                    q.popleft()
                if len(q) >= self.inflight:
                    continue
                k = min(self.chunk, min(m[1] for m in mem.values()))
                q.append(b.step(k))
                progressed = True
                for slot in list(mem):
                    mem[slot][1] -= k
                    if mem[slot][1] == 0:
                        r = mem.pop(slot)[0]
                        self.finishing.append((key, slot, b.finish(slot), r))
            # harvest members whose finish has completed
            still = []
            for key, slot, tk, r in self.finishing:
                b = self.batches[key]
                if not b.done(tk):
                    still.append((key, slot, tk, r))
                    continue
                ek, tke, eps = b.result_stats(slot)
                r.result = {"ek": ek, "tke": tke, "eps": eps}
                if self.keep_state:
                    r.result["u"] = b.get_state(slot)
                r.done = time.perf_counter() - t0
                b.reuse(slot)
                left -= 1
                progressed = True
            self.finishing = still
            if not progressed:
                nxt = pending[0].arrival - (time.perf_counter() - t0) if (pending and realtime) else 0.0
                time.sleep(min(max(nxt, 0.0), 0.0005) if nxt > 0 else 0.0001)
        for b in self.batches.values():
            b.sync()
        makespan = time.perf_counter() - t0
        return summarize(requests, makespan, self.peak_bytes)

    def close(self):
        for b in self.batches.values():
            b.close()
        self.batches.clear()


def summarize(requests: list[Request], makespan: float, peak_bytes: int = 0) -> dict:
    lat = np.array([(r.done - r.arrival) * 1e3 for r in requests])
    pts = sum(r.points * r.steps for r in requests)
    return {"requests": len(requests), "makespan_s": makespan,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "member_steps_per_s": sum(r.steps for r in requests) / makespan,
            "mpts_rk3steps_per_s": pts / makespan / 1e6, "peak_batch_bytes": peak_bytes}


def _plain_run(r: Request) -> float:
    """Seconds of one request as a plain run: create, seed, its steps (one step
    graph replayed), statistics read back, destroy."""
    t0 = time.perf_counter()
    with Simulation(r.params) as s:
        s.init_fluid()
        if r.params.p_track_part and r.params.p_np_global > 0:
            s.init_particles()
        s.advance(r.steps, sync=True)
        s.stats(last_step=True)
    return time.perf_counter() - t0


def serial_baseline(requests: list[Request]) -> dict:
    """Serial plain runs of the whole trace, every run timed: one untimed run of each
    batch class first (library set-up of that class's kernels), then each request as a
    plain run (create, seed, its steps, statistics, destroy), one after another; the
    sum of those times is what the trace takes served one run at a time."""
    seen: set = set()
    secs = 0.0
    by_size: dict[int, float] = collections.defaultdict(float)   # serial seconds per grid size
    for r in requests:
        k = class_key(r.params) + (r.steps,)
        if k not in seen:
            _plain_run(r)
            seen.add(k)
        t = _plain_run(r)
        secs += t
        by_size[r.params.nodes_x] += t
    pts = sum(r.points * r.steps for r in requests)
    return {"requests": len(requests), "runs_timed": len(requests), "classes": len(seen), "seconds": secs,
            "member_steps_per_s": sum(r.steps for r in requests) / secs, "mpts_rk3steps_per_s": pts / secs / 1e6,
            "seconds_by_size": {str(n): by_size[n] for n in sorted(by_size)}}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--requests", type=int, default=2000)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--load", type=float, default=0.8, help="arrival rate as a fraction of measured capacity")
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--variants", default="fp64,fp32_mixed")
    ap.add_argument("--capacity-sample", type=int, default=1000,
                    help="requests of the saturating run that measures capacity (the drain at its end "
                         "is a smaller share of a larger sample)")
    ap.add_argument("--tune-cache", default=None)
    ap.add_argument("--retune", action="store_true", help="measure every class's capacity afresh (not from the "
                                                          "measured table)")
    ap.add_argument("--seed", type=int, default=7)
    a = ap.parse_args(argv)
    variants = tuple(a.variants.split(","))
    budget = int(a.budget_gb * (1 << 30))
    caps = autotune(cache=a.tune_cache, start=None if a.retune else MEASURED_TABLE)
    # capacity: a saturating run (everything arrives at once) on a sample of the trace
    sample = make_trace(a.capacity_sample, seed=a.seed + 1, rate=None, steps=a.steps, variants=variants)
    srv = Server(budget, caps)
    sat = srv.run(sample, realtime=False)
    srv.close()
    capacity_rps = sat["requests"] / sat["makespan_s"]
    # the trace: Poisson arrivals at `load` x capacity
    rate = a.load * capacity_rps / len(variants)          # requests/s (each request runs every variant)
    trace = make_trace(a.requests, seed=a.seed, rate=rate, steps=a.steps, variants=variants)
    srv = Server(budget, caps)
    res = srv.run(trace, realtime=True)
    srv.close()
    base = serial_baseline(trace)
    out = {"trace": {"requests": a.requests, "runs": len(trace), "variants": list(variants), "steps": a.steps,
                     "arrival_rate_per_s": rate, "load": a.load, "budget_gb": a.budget_gb},
           "capacity": {"runs_per_s": capacity_rps, "saturated": sat},
           "served": res, "serial": base,
           "speedup_vs_serial": res["mpts_rk3steps_per_s"] / base["mpts_rk3steps_per_s"],
           "saturated_vs_serial": sat["mpts_rk3steps_per_s"] / base["mpts_rk3steps_per_s"],
           "batch_capacity": {k: v["best"] for k, v in caps.items()},
           "x_lines_per_warp": {k: v.get("xlpw", 0) for k, v in caps.items()}}
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
