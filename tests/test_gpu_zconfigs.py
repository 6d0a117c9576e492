"""Parity of the CUDA RK3 step with the CPU oracle at the sizes of the five benchmark
configurations, through the C-ABI (these take the longest of the GPU tests and sort
after the small ones):

* 64^3 decaying isotropic turbulence: u after 1, 10 and 100 steps (1e-10), E(k) and
  epsilon at every one of 100 steps (1e-8);
* 256^3 forced isotropic turbulence with 2^20 tracers: u and the forcing after 1 and
  10 steps, particle positions after 10 steps (1e-10), E(k) and epsilon;
* 512^3 homogeneous shear (BF-rot, B110 = 2, 2^18 tracers): 2 steps;
* 128^3 homogeneous shear with B110 = 2 at dt = 0.002, across its first remesh;
* 1024^3 forced flow: the FP32-mixed form against the FP64 form of the same seed on
  the same GPU (the FP64 form is the reference for this form at this size), 3 steps;
* the CFL-driven time steps (RK3_TIMESTEP_CFL, and RK3_TIMESTEP_DECIDE for isotropic
  flow, both branches of its cap), src/pf_rk3.f90:3852-3948.

Both sides start from the same state (the seeded GPU field copied to the oracle).
"""
import numpy as np
import pytest

from helpers import divergence, rel_l2, rel_l2_fields

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _periodic_maxdiff(a, b, period=2 * np.pi):
    d = np.abs(a - b)
    return float(np.minimum(d, period - d).max())


def _pair_from_gpu(pandora, p, particles=False):
    import oracle as O
    s = pandora.Simulation(p)
    s.init_fluid()
    o = O.Oracle(p)
    o.set_state(s.get_state())
    if particles:
        s.init_particles()
        o.set_particles(*s.get_particles())
    return o, s


def test_config0_decay_64_100_steps(gpu_lib):
    p = gpu_lib.workload_params("iso_decay", 64)
    assert (p.f_nu, p.rk3_dt, p.tsteps) == (0.01, 0.005, 100)
    o, s = _pair_from_gpu(gpu_lib, p)
    t = 0.0
    worst_e = worst_eps = 0.0
    for step in range(1, 101):
        ek_g, tke_g, eps_g, _ = s.stats()
        ek_o, tke_o, eps_o = o.stats()
        worst_e = max(worst_e, rel_l2(ek_g, ek_o))
        worst_eps = max(worst_eps, abs(eps_g - eps_o) / abs(eps_o))
        assert tke_g == pytest.approx(tke_o, rel=1e-8), step
        t, dt = o.step(step, t)
        assert s.step(step) == dt
        if step in (1, 10, 100):
            e = rel_l2_fields(s.get_state(), o.get_state())
            assert e < 1e-10, (step, e)
    assert worst_e < 1e-8 and worst_eps < 1e-8, (worst_e, worst_eps)
    u = s.get_state()
    assert np.abs(divergence(p, u)).max() < 1e-13 * max(np.abs(c).max() for c in u) * 64
    s.close()
    o.close()


def test_config1_forced_256_particles(gpu_lib):
    p = gpu_lib.workload_params("iso_forced_particles", 256)
    assert p.p_np_global == 1 << 20 and p.force_kf == 2.5
    o, s = _pair_from_gpu(gpu_lib, p, particles=True)
    t = 0.0
    for step in range(1, 11):
        t, dt = o.step(step, t)
        assert s.step(step) == dt
        if step in (1, 10):
            assert rel_l2_fields(s.get_forcing(), o.get_forcing()) < 1e-13, step
            e = rel_l2_fields(s.get_state(), o.get_state())
            assert e < 1e-10, (step, e)
            xg = s.get_particles()[0]
            xo = o.get_particles(p.p_np_global)[0]
            d = _periodic_maxdiff(xg, xo)
            assert d < 1e-10, (step, d)
            ek_g, tke_g, eps_g, _ = s.stats()
            ek_o, tke_o, eps_o = o.stats()
            assert rel_l2(ek_g, ek_o) < 1e-8 and abs(eps_g - eps_o) < 1e-8 * abs(eps_o), step
    s.check_status()
    s.close()
    o.close()


def test_config2_shear_512_particles(gpu_lib):
    p = gpu_lib.workload_params("shear", 512)
    assert (p.b110, p.p_np_global, p.f_remesh_t) == (2, 1 << 18, 250)
    o, s = _pair_from_gpu(gpu_lib, p, particles=True)
    t = 0.0
    for step in (1, 2):
        t, dt = o.step(step, t)
        assert s.step(step) == dt == pytest.approx(0.002, rel=1e-15)
        e = rel_l2_fields(s.get_state(), o.get_state())
        assert e < 1e-10, (step, e)
        assert s.frame() == pytest.approx(o.frame(), rel=1e-14, abs=1e-15)
        xg = s.get_particles()[0]
        xo = o.get_particles(p.p_np_global)[0]
        d = _periodic_maxdiff(xg, xo)      # positions in the computational box [0, 2 pi)^3
        assert d < 1e-10, (step, d)
    ek_g, tke_g, eps_g, _ = s.stats()
    ek_o, tke_o, eps_o = o.stats()
    assert rel_l2(ek_g, ek_o) < 1e-8 and abs(eps_g - eps_o) < 1e-8 * abs(eps_o)
    s.check_status()
    s.close()
    o.close()


def test_shear_128_b110_2_across_first_remesh(gpu_lib):
    """B110 = 2 at dt = (0.5/S)/F_REMESH_T = 0.002: S = 50 and F_REMESH_T = 5 put the
    first remesh at step B110 * F_REMESH_T + 1 = 11."""
    p = gpu_lib.workload_params("shear", 128)
    p.f_deform_s, p.f_remesh_t = 50.0, 5
    p.p_np_global = 1 << 14
    o, s = _pair_from_gpu(gpu_lib, p, particles=True)
    t = 0.0
    for step in range(1, 13):
        t, dt = o.step(step, t)
        assert s.step(step) == dt == pytest.approx(0.002, rel=1e-15)
        if step in (1, 10, 11, 12):
            e = rel_l2_fields(s.get_state(), o.get_state())
            assert e < 1e-10, (step, e)
            assert s.frame() == pytest.approx(o.frame(), rel=1e-14, abs=1e-15), step
            ek_g, tke_g, eps_g, _ = s.stats()
            ek_o, tke_o, eps_o = o.stats()
            assert rel_l2(ek_g, ek_o) < 1e-8 and abs(eps_g - eps_o) < 1e-8 * abs(eps_o), step
    xg = s.get_particles()[0]
    xo = o.get_particles(p.p_np_global)[0]
    d = _periodic_maxdiff(xg, xo)
    assert d < 1e-10, d
    assert np.abs(divergence(p, s.get_state())).max() < 1e-13
    s.check_status()
    s.close()
    o.close()


class _DeviceArray:
    """A device buffer of the library as a torch tensor (no copy): complex values of the
    stored precision as (n, 2) reals."""

    def __init__(self, ptr, n, fp32):
        self.__cuda_array_interface__ = {"shape": (n, 2), "typestr": "<f4" if fp32 else "<f8",
                                         "data": (ptr, False), "version": 3, "strides": None}


def test_config3_mixed_1024_against_fp64(gpu_lib):
    """FP32 fields and transforms against the FP64 form of the same seed, 3 steps at
    1024^3: E(k) within 1e-4 relative (the mixed form's stated bar), u within 1e-5 relative L2,
    epsilon within 1e-4.  u is compared on the device."""
    import torch
    p = gpu_lib.workload_params("iso_forced", 1024)
    assert (p.f_nu, p.rk3_dt) == (0.0008, 0.001)
    q = p.copy()
    q.precision = gpu_lib.PREC_FP32_MIXED
    with gpu_lib.Simulation(p) as s64, gpu_lib.Simulation(q) as s32:
        for s in (s64, s32):
            s.init_fluid()
        for step in (1, 2, 3):
            assert s64.step(step) == s32.step(step)
        ek64, tke64, eps64, _ = s64.stats()
        ek32, tke32, eps32, _ = s32.stats()
        assert rel_l2(ek32, ek64) < 1e-4 and abs(eps32 - eps64) < 1e-4 * abs(eps64)
        assert tke32 == pytest.approx(tke64, rel=1e-5)
        num = den = 0.0
        for a, b in zip(s64.device_state_ptrs(), s32.device_state_ptrs()):
            x = torch.as_tensor(_DeviceArray(a, s64.modes, False), device="cuda")
            y = torch.as_tensor(_DeviceArray(b, s32.modes, True), device="cuda")
            num += float(((y.double() - x) ** 2).sum())
            den += float((x ** 2).sum())
        torch.cuda.synchronize()
        e = (num / den) ** 0.5
        assert 0.0 < e < 1e-5, e


@pytest.mark.parametrize("mode,tf", [("cfl", 0.2), ("decide", 10.0), ("decide", 0.004)])
def test_cfl_driven_time_step(gpu_lib, mode, tf):
    """RK3_TIMESTEP_CFL: dt = RK3_CFL dx / max(|u1|+|u2|+|u3|) of the stage-1 physical
    field; RK3_TIMESTEP_DECIDE (isotropic): the same, capped at FORCE_TF (tf = 10: the CFL
    branch; tf = 0.004: the cap).  Forced flow at 64^3 with tracers, 10 steps."""
    p = gpu_lib.workload_params("iso_forced_particles", 64)
    p.p_np_global = 4096
    p.rk3_timestep = gpu_lib.RK3_TIMESTEP_CFL if mode == "cfl" else gpu_lib.RK3_TIMESTEP_DECIDE
    p.rk3_cfl, p.force_tf = 0.5, tf
    o, s = _pair_from_gpu(gpu_lib, p, particles=True)
    t = 0.0
    dts = []
    for step in range(1, 11):
        t, dt = o.step(step, t)
        dtg = s.step(step)
        assert dtg == pytest.approx(dt, rel=1e-13), step
        dts.append(dt)
        if step in (1, 10):
            e = rel_l2_fields(s.get_state(), o.get_state())
            assert e < 1e-10, (step, e)
    assert s.simtime == pytest.approx(t, rel=1e-13)
    dx = 2 * np.pi / 64
    if mode == "decide" and tf < 0.01:
        assert all(d == tf for d in dts)           # the cap
    else:
        assert len(set(dts)) > 1                    # dt follows the flow
        ucfl = s.stats(last_step=True)[3]          # max |u1|+|u2|+|u3| at stage 1 of the last step
        assert dts[-1] == pytest.approx(0.5 * dx / ucfl, rel=1e-14)
    xg = s.get_particles()[0]
    xo = o.get_particles(p.p_np_global)[0]
    assert _periodic_maxdiff(xg, xo) < 1e-10
    s.close()
    o.close()
