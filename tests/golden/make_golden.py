"""Regenerates the regression fixtures in this folder from the CPU oracle.

The reference (Fortran + MPI + PETSc + FFTW) cannot be built or imported here, so
its own data pin only the known-answer test in kat_nonlinear.json; these fixtures
freeze the oracle's output on small cases (16^3 and 24^3) so that any later change
of the oracle or of the CUDA path is caught against fixed numbers.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "pandora-2.0_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from pandora.params import workload_params  # noqa: E402


def case(name, n, steps, np_particles=0):
    p = workload_params(name, n)
    if np_particles:
        p.p_np_global = np_particles
    else:
        p.p_track_part = 0
    o = O.Oracle(p)
    o.init_fluid()
    u0 = o.get_state()
    if np_particles:
        o.init_particles()
    x0 = o.get_particles(np_particles)[0] if np_particles else np.zeros((0, 3))
    t = 0.0
    for s in range(1, steps + 1):
        t, dt = o.step(s, t)
    ek, tke, eps = o.stats()
    out = dict(u0=np.stack(u0), u=np.stack(o.get_state()), rk=np.stack(o.get_rk()), ek=ek, tke=tke, eps=eps,
               simtime=t, x0=x0, x=o.get_particles(np_particles)[0] if np_particles else np.zeros((0, 3)),
               forcing=np.stack(o.get_forcing()))
    np.savez_compressed(os.path.join(HERE, f"{name}_{n}_{steps}.npz"), **out)


if __name__ == "__main__":
    case("iso_decay", 16, 3)
    case("iso_forced_particles", 24, 3, np_particles=64)
    print("written")
