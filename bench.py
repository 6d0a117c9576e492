"""Benchmark of the PANDORA 2.0 RK3 time step on B200.

Workload (default): homogeneous shear at 512^3 in the Rogallo frame (BF-rot form,
F_TYPE = F_SHEAR_DNS), lab box 4pi x 2pi x 2pi (B110 = 2), S = 1, nu = 0.005,
dt = (0.5/S)/F_REMESH_T = 0.002, FP64, 2^18 tracers with 4th-order interpolation
advanced at every stage; synthetic seeded initial field (Ahmed/Elghobashi spectrum,
kp = 4, u0 = 0.5).  A "step" is one full RK3 step (three stages, statistics at
stage 1, particles, the remesh check).  ``--workload iso_forced_particles --n 256``
gives the forced isotropic case with 2^20 tracers.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas, one process per GPU (launched by torchrun):
the path has no exchange step on one field, so there is no collective in the
data path; the barrier and the max-over-ranks timing use torch.distributed.
Prints ONE JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "pandora-2.0_b200"))

METRIC = "Mpts·RK3steps/s"
WORKLOAD = "shear"
# DRAM traffic (read + write bytes) of one launch of a pass in stages 2-3, from ncu
# captures of dram__bytes_read.sum + dram__bytes_write.sum: (workload, N, form) -> pass ->
# bytes.  256^3: captured at full size.  512^3: each 512-point pass captured on a case
# whose other two axes are 128 points (512x128x128, 128x512x128, 128x128x512, tracers at
# the same density) and scaled to the full grid by the ratio of algorithmic bytes; the
# commands and the raw figures are summarised under profiles/.
NCU_TRAFFIC_BYTES = {
    ("iso_forced_particles", 256, "fp64_plain"): {
        "zpass_inv": 432157440, "ypass_inv": 862682752, "xpass_nl": 1177856256, "ypass_fwd": 417905024,
        "zpass_fwd_update": 261682560 + 549060736, "particles": 605924864},
    ("shear", 512, "fp64_plain"): {
        "zpass_inv": 3199086129, "ypass_inv": 7047367930, "xpass_nl": 8904337408, "ypass_fwd": 3324333151,
        "zpass_fwd_update": 1928149719 + 3921155948, "particles": 1473873920},
}
# Seconds of host work the reference arm spends on its timed steps at most (the
# whole arm, warm-up and set-up included, stays within a few minutes).
REF_BUDGET_S = 100.0


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--n", "--grid", dest="n", type=int, default=None,
                    help="grid points per direction (default: the workload's own, 512 for shear)")
    ap.add_argument("--np", "--particles", dest="np", type=int, default=None,
                    help="tracers (default: the workload's own, 2^18 for shear)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32_mixed"],
                    help="fp32_mixed: FP32 fields and transforms, FP64 bookkeeping (our arm only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def _params(a, fp64=False):
    from pandora.params import PREC_FP32_MIXED, PREC_FP64, workload_params
    p = workload_params(a.workload, a.n)
    if p.p_track_part and a.np is not None:
        p.p_np_global = a.np
    p.precision = PREC_FP32_MIXED if (a.precision == "fp32_mixed" and not fp64) else PREC_FP64
    return p


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Ranks:
    """The replicas' only cross-rank traffic: a barrier around the timed region and the
    max over ranks of each timing (NCCL on GPUs; gloo with device "cpu" in the tests)."""

    def __init__(self, backend: str = "nccl", device: str = "cuda", timeout_s: int = 120):
        self.ws, self.rank, self.local = _dist()
        self.device = device
        if self.ws > 1:
            import torch.distributed as dist
            from datetime import timedelta
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))

    def barrier(self):
        if self.ws > 1:
            import torch.distributed as dist
            dist.barrier()

    def max(self, x: float) -> float:
        if self.ws == 1:
            return x
        import torch
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.ws > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


def replica_seeds(p, rank: int):
    """Each replica runs its own member of the ensemble: same workload, own seeds."""
    p.seed_fluid = 1 + rank
    p.seed_force = 1000 + rank
    p.seed_particles = 2000 + rank
    return p


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = sorted(v for v in (num(r[1]) for r in self.rows) if v is not None)
        smax = max((v for v in (num(r[2]) for r in self.rows) if v is not None), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(self.rows)}


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _oracle(p):
    """The oracle (CPU restatement of the reference, OpenMP over the host cores) on the
    workload's seeded initial state."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    o = O.Oracle(p)
    o.init_fluid()
    if p.p_track_part:
        o.init_particles()
    return O, o


def cpu_baseline(p):
    """One warm RK3 step of the same workload on the host: one step untimed (first touch
    of every array, thread pool start), then one step timed.
    Returns (Mpts*steps/s, cores, secs of the timed step)."""
    O, o = _oracle(p)
    t, _ = o.step(1, 0.0)
    t0 = time.perf_counter()
    o.step(2, t)
    secs = time.perf_counter() - t0
    npts = p.nodes_x * p.nodes_y * p.nodes_z
    o.close()
    return npts / secs / 1e6, O.threads(), secs


def run_reference(a, p):
    """The reference's algorithm on the host cores (the oracle's OpenMP C restatement:
    the Fortran + MPI + PETSc + FFTW reference has no toolchain on this image).  Times
    whole RK3 steps: up to W warm-up steps (at least one, at most three), then K timed
    steps or as many as fit in REF_BUDGET_S seconds, whichever is fewer; the line reports
    the counts actually run."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    O, o = _oracle(p)
    npts = p.nodes_x * p.nodes_y * p.nodes_z
    t = 0.0
    step = 1
    n_warm = max(1, min(a.warmup, 3))
    w0 = time.perf_counter()
    for _ in range(n_warm):
        t, _ = o.step(step, t)
        step += 1
    per = (time.perf_counter() - w0) / n_warm
    n_timed = max(1, min(a.steps, int(REF_BUDGET_S // max(per, 1e-9))))
    t0 = time.perf_counter()
    for _ in range(n_timed):
        t, _ = o.step(step, t)
        step += 1
    secs = time.perf_counter() - t0
    o.close()
    value = npts * n_timed / secs / 1e6
    cores = O.threads()
    sample = (f"{n_timed} whole RK3 steps (3 stages each) of the full workload after {n_warm} warm-up "
              f"step(s), OpenMP C restatement of the reference's algorithm (oracle/pandora_oracle.c) on "
              f"{cores} threads of {cpu_model()}; the reference binary (Fortran+MPI+PETSc+FFTW) has no "
              f"toolchain on this image")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": a.gpus,
        "steps": n_timed, "warmup": n_warm, "ms_per_step": 1e3 * secs / n_timed,
        "requested": {"steps": a.steps, "warmup": a.warmup, "budget_s": REF_BUDGET_S},
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Rogallo field, seeded tracers)",
        "config": _config(a, p),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": "port", "cpu": cpu_model(),
                         "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def form_key(p) -> str:
    return "fp32_mixed" if p.precision == 1 else "fp64_plain"


def _config(a, p):
    npart = int(p.p_np_global) if p.p_track_part else 0
    if p.f_type == 2:
        dt = 0.5 / p.f_deform_s / p.f_remesh_t
        form_name = {1: "BF-rot", 2: "R-conv", 3: "R-rot"}.get(p.ns_deformed, "?")
        first = p.b110 * p.f_remesh_t + 1
        phys = (f"homogeneous shear S={p.f_deform_s} (Rogallo frame, {form_name}), box "
                f"{2 * p.b110}pi x 2pi x 2pi (B110={p.b110}), nu={p.f_nu}, dt=(0.5/S)/F_REMESH_T={dt:g} "
                f"(remesh at step {first} and every {2 * p.b110 * p.f_remesh_t} steps after), no forcing")
    elif p.force_stop > 0:
        phys = f"OU forcing |k|<={p.force_kf}, nu={p.f_nu}, dt={p.rk3_dt}"
    else:
        phys = f"decaying, nu={p.f_nu}, dt={p.rk3_dt}"
    ws = (6 * 16 * (p.nodes_x // 3 + 8) * p.nodes_y * p.nodes_z) / 1e9
    form = "FP32-mixed" if p.precision == 1 else "FP64 plain"
    return {"workload": f"{a.workload} {p.nodes_x}^3 {form}, {phys}, {npart} tracers (order {p.p_interp_order})",
            "grid": [p.nodes_x, p.nodes_y, p.nodes_z], "nu": p.f_nu,
            "particles": npart, "form": "fp32_mixed" if p.precision == 1 else "fp64_plain",
            "parallelism": f"replicas x{a.gpus}",
            "l2": f"no flush needed: each pass streams > 126 MB (y-pencil buffer alone {ws:.2f} GB)"}


def _step_model(p, ms_per_step, peak):
    ki, kj, kk = p.nodes_x // 3, p.nodes_y // 3, p.nodes_z // 3
    S = (ki + 1) * (2 * kj + 1) * (2 * kk + 1)
    Z = (ki + 1) * (2 * kj + 1) * p.nodes_z
    Y = (ki + 1) * p.nodes_y * p.nodes_z
    R = p.nodes_x * p.nodes_y * p.nodes_z
    w = 4.0 if p.precision == 1 else 8.0      # real word of the fields (FP32-mixed: 4 B)
    b = 3 * 2 * w * (15 * S + 18 * Z + 18 * Y) + 2 * w * 3 * S
    if p.p_track_part and p.p_np_global > 0:
        # physical velocity in the fields' word, particle state in FP64
        b += 3 * (6 * R * w + 18 * 8.0 * p.p_np_global)
    achieved = b / (ms_per_step / 1e3) / 1e9
    return {"bytes_per_step": b, "achieved": achieved, "frac": achieved / peak,
            "model": f"3 stages x {2 * w:.0f} B x (15S + 18Z + 18Y) + stats 3S + particles 3 x (6R x {w:.0f} B + 18Np x 8 B)"}


def run_ours(a, p):
    import torch
    import pandora

    ws, rank, local = _dist()
    torch.cuda.set_device(local if ws > 1 else 0)
    ranks = Ranks("nccl", "cuda")
    dev = torch.cuda.current_device()
    barrier = ranks.barrier
    max_over_ranks = ranks.max
    replica_seeds(p, rank)
    sim = pandora.Simulation(p)
    sim.init_fluid()
    if p.p_track_part:
        sim.init_particles()
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    npts = p.nodes_x * p.nodes_y * p.nodes_z

    # warm-up with event pairs around every pass inside the step graph, to find the
    # dominant pass; the timed region then carries the pair around that pass only
    # (6 event nodes per step), whose durations in the last timed step give the roofline
    sim.set_pass_timing(0x3F)
    sim.advance(max(a.warmup, 3), sync=True)
    warm = sim.pass_times()
    # the dominant pass; its event pairs of stages 2 and 3 time it with the GPU to itself
    # (the only second-stream work, the particle sort, runs beside stage 1)
    solo = [1, 2, 3, 4, 5]
    dom_pid = max(solo, key=lambda q: warm[1:, q - 1].mean())
    sim.set_pass_timing(1 << (dom_pid - 1))
    sim.advance(3, sync=True)
    sim.check_status()

    # ---- device-resident timing ----
    sampler = ClockSampler(dev)
    sampler.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.advance(a.steps, sync=False)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    live = sim.pass_times()          # [stage][pass] ms of the last timed step
    sim.check_status()

    # ---- end to end through the C-ABI: one synchronous g_RK3Calc call per step
    # (host scalars tstep/simtime in, dt/simtime out) plus the step's statistics
    # (E(k), tke, eps, ucfl) read back to the host ----
    n_e2e = max(1, min(a.steps, 200))
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        sim.step()
        sim.stats(last_step=True)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    sampler.stop()
    clocks = sampler.summary()

    # ---- roofline of the dominant pass: its launches in the last timed step
    # (CUDA event pairs recorded inside the step graph, stages 2 and 3, whose
    # traffic pass_bytes counts); each pass also timed alone for reference ----
    peak, peak_kind = _peaks()
    passes = {1: "zpass_inv", 2: "ypass_inv", 3: "xpass_nl", 4: "ypass_fwd", 5: "zpass_fwd_update",
              6: "particles"}
    per_pass_live = {}
    for pid, name in passes.items():
        v = live[1:, pid - 1] if pid == dom_pid else warm[1:, pid - 1]
        if (v > 0).all():
            b = sim.pass_bytes(pid)
            d = float(v.mean()) / 1e3
            per_pass_live[name] = {"ms": d * 1e3, "gbs": b / d / 1e9}
    per_pass = {}
    reps = 20
    for pid, name in passes.items():
        if pid == 6 and not (p.p_track_part and p.p_np_global > 0):
            continue
        sim.profile_pass(pid, 2)
        q0 = torch.cuda.Event(enable_timing=True)
        q1 = torch.cuda.Event(enable_timing=True)
        q0.record(stream)
        sim.profile_pass(pid, reps)
        q1.record(stream)
        torch.cuda.synchronize()
        dur = q0.elapsed_time(q1) / reps / 1e3
        b = sim.pass_bytes(pid)
        per_pass[name] = {"ms": dur * 1e3, "gbs": b / dur / 1e9, "bytes": b}
    traffic = NCU_TRAFFIC_BYTES.get((a.workload, p.nodes_x, form_key(p)), {})
    for name, v in per_pass.items():
        if name in traffic:
            v["traffic_over_alg"] = traffic[name] / v["bytes"]
    src = per_pass_live if per_pass_live else per_pass
    dom = passes[dom_pid] if passes[dom_pid] in src else max(src, key=lambda k: src[k]["ms"])
    dom_gbs = src[dom]["gbs"]
    roofline = {"bound": "hbm", "kernel": dom, "achieved": dom_gbs, "peak": peak, "unit": "GB/s",
                "frac": dom_gbs / peak, "peak_kind": f"{peak_kind} (burst copy)",
                "timed": ("dominant pass (of those with the GPU to themselves): event pair in the step graph, stages 2-3 of the last timed step; "
                          "other passes: the same in the last warm-up step") if per_pass_live
                         else "alone, 20 back-to-back launches",
                "traffic": traffic.get(dom),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch (table in bench.py)"
                                  if traffic else None,
                "per_pass": {k: {"ms": round(v["ms"], 4), "GB/s": round(v["gbs"], 1)} for k, v in src.items()},
                "per_pass_alone": {k: {"ms": round(v["ms"], 4), "GB/s": round(v["gbs"], 1),
                                       **({"traffic/alg": round(v["traffic_over_alg"], 3)}
                                          if "traffic_over_alg" in v else {})}
                                   for k, v in per_pass.items()}}
    launches = sim.launches_per_step()
    value = npts * a.steps * ws / (ms / 1e3) / 1e6
    e2e_value = npts * n_e2e * ws / e2e_s / 1e6
    kk = sim.kkmax
    d2h = 48 + 8 * (2 * (kk + 1) + 3) + 48
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if p.precision == 1 else "f64",
        "data": "synthetic (seeded Rogallo field, seeded tracers)",
        "config": _config(a, p),
        "clocks": clocks,
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": 48, "d2h_bytes_per_step": d2h,
                "steps": n_e2e, "what": "pandora_rk3_step + pandora_last_step_stats per step, host wall clock"},
        "gpu_launches": launches * a.steps,
        "roofline": roofline,
        "step_model_gbs": None,
    }
    # whole-step algorithmic bytes: the fused 5-pass model (per stage 15 S + 18 Z + 18 Y
    # complex words; particles add 6 R + 18 Np words per stage; stage-1 stats read 3 S)
    line["step_model_gbs"] = _step_model(p, ms / a.steps, peak)
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        v, cores, secs = cpu_baseline(_params(a, fp64=True))
        line["cpu_baseline"] = {"value": v, "unit": METRIC, "cores": cores, "kind": "port", "cpu": cpu_model(),
                                "sample": f"one warm RK3 step (3 stages, after one untimed step) of the same "
                                          f"workload in FP64 on {cores} threads of the host, {secs:.1f} s, OpenMP C "
                                          f"restatement of the reference's algorithm (oracle/pandora_oracle.c)"}
    sim.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def main():
    a = _args()
    if a.impl == "reference":
        return run_reference(a, _params(a, fp64=True))
    p = _params(a)
    return run_ours(a, p)


if __name__ == "__main__":
    sys.exit(main())
