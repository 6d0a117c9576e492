"""The FP32-mixed form (PANDORA_PREC_FP32_MIXED) against the FP64 oracle.

Fields, transforms and the nonlinear term run in FP32; the boundary stays FP64.
The bars of this form: E(k) within 1e-4 relative of the FP64
oracle, plus u within 1e-5 relative L2, epsilon within 1e-4 and particle positions
within 1e-6 (about 10 FP32 roundings of O(1) quantities over a few steps).
"""
import numpy as np
import pytest

from helpers import rel_l2, rel_l2_fields

pytestmark = pytest.mark.gpu


def _mixed(pandora, p):
    import oracle as O
    o = O.Oracle(p)
    o.init_fluid()
    q = pandora.Params.from_buffer_copy(p)
    q.precision = pandora.PREC_FP32_MIXED
    s = pandora.Simulation(q)
    s.set_state(o.get_state())
    return o, s


def test_state_round_trip_rounds_to_fp32(gpu_lib):
    p = gpu_lib.workload_params("iso_decay", 32)
    o, s = _mixed(gpu_lib, p)
    u = o.get_state()
    back = s.get_state()
    for a, b in zip(u, back):
        want = a.real.astype(np.float32).astype(np.float64) + 1j * a.imag.astype(np.float32).astype(np.float64)
        assert np.array_equal(b, want)
    s.close()


@pytest.mark.parametrize("n", [24, 32, 64])
def test_mixed_nonlinear(gpu_lib, n):
    p = gpu_lib.workload_params("iso_decay", n)
    o, s = _mixed(gpu_lib, p)
    e = rel_l2_fields(s.nonlinear(), o.nonlinear())
    s.close()
    assert e < 1e-5, e


@pytest.mark.parametrize("dims", [(64, 512, 16), (64, 16, 512), (512, 16, 16), (16, 1024, 16),
                                  (16, 16, 1024), (1024, 16, 16), (256, 16, 32), (48, 192, 96),
                                  (80, 112, 160), (640, 16, 56), (16, 896, 40)])
def test_mixed_nonlinear_every_tile_shape(gpu_lib, dims):
    """Long lines in each direction of the FP32 form, including tiles of 16 lines
    whose last tile is partial (nkip = 24 at nx = 64)."""
    p = gpu_lib.workload_params("iso_decay", 32)
    p.nodes_x, p.nodes_y, p.nodes_z = dims
    o, s = _mixed(gpu_lib, p)
    e = rel_l2_fields(s.nonlinear(), o.nonlinear())
    s.close()
    assert e < 1e-5, e


def test_mixed_decay_10_steps(gpu_lib):
    p = gpu_lib.workload_params("iso_decay", 64)
    o, s = _mixed(gpu_lib, p)
    t = 0.0
    for step in range(1, 11):
        t, _ = o.step(step, t)
        s.step(step)
    eu = rel_l2_fields(s.get_state(), o.get_state())
    ek_g, tke_g, eps_g, _ = s.stats()
    ek_o, tke_o, eps_o = o.stats()
    s.close()
    assert eu < 1e-5, eu
    assert rel_l2(ek_g, ek_o) < 1e-4 and abs(eps_g - eps_o) / abs(eps_o) < 1e-4


def test_mixed_forced_particles(gpu_lib):
    p = gpu_lib.workload_params("iso_forced_particles", 32)
    p.p_np_global = 2048
    o, s = _mixed(gpu_lib, p)
    s.init_particles()
    o.set_particles(*s.get_particles())
    t = 0.0
    for step in range(1, 6):
        t, _ = o.step(step, t)
        s.step(step)
    assert rel_l2_fields(s.get_forcing(), o.get_forcing()) < 1e-13   # forcing stays FP64
    assert rel_l2_fields(s.get_state(), o.get_state()) < 1e-5
    xg = s.get_particles()[0]
    xo = o.get_particles(p.p_np_global)[0]
    d = np.abs(xg - xo)
    d = np.minimum(d, 2 * np.pi - d)
    assert d.max() < 1e-6, d.max()
    s.check_status()
    s.close()


def test_mixed_shear_across_remesh(gpu_lib):
    """BF-rot shear at 32^3 with a remesh inside the run (f_remesh_t = 2: every 4 steps)."""
    p = gpu_lib.workload_params("shear", 32)
    p.p_track_part = 0
    p.f_remesh_t = 2
    o, s = _mixed(gpu_lib, p)
    t = 0.0
    for step in range(1, 7):
        t, _ = o.step(step, t)
        s.step(step)
    e = rel_l2_fields(s.get_state(), o.get_state())
    s.close()
    assert e < 1e-4, e


@pytest.mark.parametrize("form", [2, 3])
def test_mixed_rogallo_across_remesh(gpu_lib, form):
    """R-conv (2) and R-rot (3) shear forms in FP32 at 32^3 across a remesh."""
    p = gpu_lib.workload_params("shear", 32)
    p.p_track_part = 0
    p.f_remesh_t = 2
    p.ns_deformed = form
    o, s = _mixed(gpu_lib, p)
    t = 0.0
    for step in range(1, 7):
        t, _ = o.step(step, t)
        s.step(step)
    e = rel_l2_fields(s.get_state(), o.get_state())
    s.close()
    assert e < 1e-4, e


def test_mixed_error_module_small(gpu_lib):
    """pandora.mixed_error on a small case: both forms from one seed, errors stated."""
    from pandora import mixed_error
    p = gpu_lib.workload_params("iso_forced", 32)
    r = mixed_error.compare(p, 6)
    assert r["rel_l2_u"] < 1e-5 and r["rel_l2_ek"] < 1e-4 and r["rel_eps"] < 1e-4, r
    assert r["ms_per_step_fp64"] > 0 and r["ms_per_step_fp32_mixed"] > 0


def test_mixed_dealias_spherical(gpu_lib):
    p = gpu_lib.workload_params("iso_decay", 32)
    p.dealiasing = 2
    o, s = _mixed(gpu_lib, p)
    t = 0.0
    for step in range(1, 11):
        t, _ = o.step(step, t)
        s.step(step)
    eu = rel_l2_fields(s.get_state(), o.get_state())
    s.close()
    assert eu < 1e-5, eu


def test_mixed_realspace_stats(gpu_lib):
    p = gpu_lib.workload_params("iso_decay", 32)
    o, s = _mixed(gpu_lib, p)
    g, r = s.realspace_sums(), o.realspace_sums()
    s.close()
    np.testing.assert_allclose(g, r, rtol=1e-5)

