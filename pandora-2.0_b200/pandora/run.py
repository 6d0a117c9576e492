"""Run a named workload for a few steps on any grid: the driver loop of a plain
simulation (create, seed, advance, statistics), for profiling a kernel on a case
smaller than the benchmark's.

    python -m pandora.run --workload shear --nodes 512 128 128 --steps 3
"""
from __future__ import annotations

import argparse
import sys

from .params import PREC_FP32_MIXED, PREC_FP64, workload_params
from .rk3 import Simulation


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", default="shear")
    ap.add_argument("--nodes", type=int, nargs=3, metavar=("NX", "NY", "NZ"), default=(64, 64, 64))
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--np", type=int, default=0, help="tracers (0: none)")
    ap.add_argument("--precision", choices=["fp64", "fp32_mixed"], default="fp64")
    a = ap.parse_args(argv)
    p = workload_params(a.workload, a.nodes[0])
    p.nodes_x, p.nodes_y, p.nodes_z = a.nodes
    p.p_track_part, p.p_np_global = (1, a.np) if a.np > 0 else (0, 0)
    p.precision = PREC_FP32_MIXED if a.precision == "fp32_mixed" else PREC_FP64
    with Simulation(p) as s:
        s.init_fluid()
        if a.np > 0:
            s.init_particles()
        s.advance(a.steps)
        ek, tke, eps, _ = s.stats()
        s.check_status()
    print(f"{a.workload} {a.nodes[0]}x{a.nodes[1]}x{a.nodes[2]} {a.precision}: {a.steps} steps, tke {tke:.6e}, eps {eps:.6e}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
