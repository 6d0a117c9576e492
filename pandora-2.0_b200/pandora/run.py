"""Run a named workload for a few steps on any grid: the driver loop of a plain
simulation (create, seed, advance, statistics), for profiling a kernel on a case
smaller than the benchmark's.

    python -m pandora.run --workload shear --nodes 512 128 128 --steps 3
    python -m pandora.run --workload shear --nodes 512 512 512 --form r-conv --pass-times
    python -m pandora.run --workload iso_decay --nodes 32 32 32 --batch 32 --steps 20

``--form`` picks the shear formulation (NS_DEFORMED); ``--pass-times`` times every
pass of the last step with CUDA event pairs and prints them (ms, stage x pass);
``--batch CAP`` runs a batch of CAP members of the workload (own seeds) instead of one
simulation and prints its member-steps/s.
"""
from __future__ import annotations

import argparse
import sys

from .params import NS_BF_ROT, NS_R_CONV, NS_R_ROT, PREC_FP32_MIXED, PREC_FP64, workload_params

FORMS = {"bf-rot": NS_BF_ROT, "r-conv": NS_R_CONV, "r-rot": NS_R_ROT}
PASSES = ("zpass_inv", "ypass_inv", "xpass", "ypass_fwd", "zpass_fwd_update", "particles")
from .rk3 import Simulation


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", default="shear")
    ap.add_argument("--nodes", type=int, nargs=3, metavar=("NX", "NY", "NZ"), default=(64, 64, 64))
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--np", type=int, default=0, help="tracers (0: none)")
    ap.add_argument("--precision", choices=["fp64", "fp32_mixed"], default="fp64")
    ap.add_argument("--form", choices=sorted(FORMS), default="bf-rot", help="shear formulation")
    ap.add_argument("--pass-times", action="store_true", help="time each pass of the last step")
    ap.add_argument("--batch", type=int, default=0, help="members of a batch (0: one simulation)")
    ap.add_argument("--xlpw", type=int, default=0, help="x lines per warp (x_lines_per_warp; 0: the library's choice)")
    a = ap.parse_args(argv)
    p = workload_params(a.workload, a.nodes[0])
    p.nodes_x, p.nodes_y, p.nodes_z = a.nodes
    p.p_track_part, p.p_np_global = (1, a.np) if a.np > 0 else (0, 0)
    p.precision = PREC_FP32_MIXED if a.precision == "fp32_mixed" else PREC_FP64
    p.ns_deformed = FORMS[a.form]
    p.x_lines_per_warp = a.xlpw
    if a.batch > 0:
        return _run_batch(p, a)
    with Simulation(p) as s:
        s.init_fluid()
        if a.np > 0:
            s.init_particles()
        if a.pass_times and a.steps > 1:
            s.advance(a.steps - 1)
        if a.pass_times:
            s.set_pass_timing(0x3F)
            s.advance(1)
            t = s.pass_times()
            s.set_pass_timing(0)
            for name, col in zip(PASSES, t.T):   # -1: not timed (no particles)
                if (col < 0).all():
                    continue
                print(f"{name:10s} " + " ".join(f"{v:8.3f}" for v in col) + f"   sum {col[col > 0].sum():8.3f} ms")
            print(f"step (sum of passes) {t[t > 0].sum():.3f} ms")
        else:
            import time
            s.advance(1)
            t0 = time.perf_counter()
            s.advance(a.steps - 1 if a.steps > 1 else 1)
            ms = (time.perf_counter() - t0) * 1e3 / max(a.steps - 1, 1)
            print(f"{ms:.4f} ms per step (host clock over {max(a.steps - 1, 1)} steps)")
        ek, tke, eps, _ = s.stats()
        s.check_status()
    print(f"{a.workload} {a.nodes[0]}x{a.nodes[1]}x{a.nodes[2]} {a.precision}: {a.steps} steps, tke {tke:.6e}, eps {eps:.6e}")
    return 0


def _run_batch(p, a) -> int:
    import time
    from .batch import Batch
    with Batch(p, a.batch) as b:
        for k in range(a.batch):
            q = p.copy()
            q.seed_fluid, q.seed_force, q.seed_particles = 1 + k, 1000 + k, 2000 + k
            b.admit(q)
        b.step(1)
        b.sync()
        t0 = time.perf_counter()
        b.step(a.steps)
        b.sync()
        secs = time.perf_counter() - t0
    print(f"{a.workload} {a.nodes[0]}x{a.nodes[1]}x{a.nodes[2]} {a.precision} batch of {a.batch}: "
          f"{a.steps} steps, {a.batch * a.steps / secs:.0f} member-steps/s")
    return 0


if __name__ == "__main__":
    sys.exit(main())
