"""Parity of the CUDA RK3 step with the CPU oracle, through the C-ABI.

Tolerances (FP64 plain form): u within 1e-10 relative L2 after 1 and 10 steps,
E(k) and epsilon within 1e-8 over 100 steps, particle positions within 1e-10
after 10 steps, div u at round-off.  Both sides start from the same state.
"""
import numpy as np
import pytest

from helpers import divergence, rel_l2, rel_l2_fields

pytestmark = pytest.mark.gpu


def _pair(pandora, p, init="oracle"):
    import oracle as O
    o = O.Oracle(p)
    s = pandora.Simulation(p)
    if init == "oracle":
        o.init_fluid()
        s.set_state(o.get_state())
    else:
        s.init_fluid()
        o.set_state(s.get_state())
    return o, s


def test_nonlinear_known_answer(gpu_lib):
    """src/ptf_rk3.f90:1115-1191: L1 norms of NL-hat = 3/4, 9/8, 11/8."""
    import oracle as O
    p = gpu_lib.default_params(32)
    o = O.Oracle(p)
    o.init_taylor_green_reverse()
    with gpu_lib.Simulation(p) as s:
        s.set_state(o.get_state())
        nl = s.nonlinear()
    l1 = [float(np.abs(c.real).sum() + np.abs(c.imag).sum()) for c in nl]
    assert np.allclose(l1, [0.75, 1.125, 1.375], rtol=1e-12, atol=0), l1
    assert rel_l2_fields(nl, o.nonlinear()) < 1e-13


@pytest.mark.parametrize("n", [16, 24, 32, 48, 64])
def test_nonlinear_matches_oracle(gpu_lib, n):
    p = gpu_lib.workload_params("iso_decay", n)
    o, s = _pair(gpu_lib, p)
    nl_g = s.nonlinear()
    nl_o = o.nonlinear()
    s.close()
    assert rel_l2_fields(nl_g, nl_o) < 1e-13


def test_nonlinear_anisotropic_grid(gpu_lib):
    p = gpu_lib.workload_params("iso_decay", 32)
    p.nodes_x, p.nodes_y, p.nodes_z = 32, 48, 64
    o, s = _pair(gpu_lib, p)
    e = rel_l2_fields(s.nonlinear(), o.nonlinear())
    s.close()
    assert e < 1e-13


@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("n", [40, 56, 80, 96, 112, 128, 160, 192, 224, 256, 320, 384, 448, 512, 640, 768, 896, 1024])
def test_nonlinear_every_length(gpu_lib, n, axis):
    """Every supported transform length along each axis (x pass, y passes, z passes),
    the other two axes 16 points long; the lengths 2^a x {1, 3, 5, 7} of the reference's
    size rule (src/pg_domain.f90:274-292)."""
    p = gpu_lib.workload_params("iso_decay", 32)
    dims = [16, 16, 16]
    dims[axis] = n
    p.nodes_x, p.nodes_y, p.nodes_z = dims
    o, s = _pair(gpu_lib, p)
    e = rel_l2_fields(s.nonlinear(), o.nonlinear())
    s.close()
    assert e < 1e-13


def test_init_fluid_matches_oracle(gpu_lib):
    import oracle as O
    p = gpu_lib.workload_params("iso_decay", 64)
    o = O.Oracle(p)
    o.init_fluid()
    with gpu_lib.Simulation(p) as s:
        s.init_fluid()
        ug = s.get_state()
    uo = o.get_state()
    assert rel_l2_fields(ug, uo) < 1e-13
    # conjugate symmetry of the i=0 plane: u(0,-j,-k) = conj u(0,j,k)
    for c in ug:
        pl = c[0]
        flip = np.conj(np.roll(pl[::-1, ::-1], 1, axis=(0, 1)))
        assert np.abs(pl - flip).max() < 1e-15


@pytest.mark.parametrize("n", [32, 64])
def test_step_parity_decay(gpu_lib, n):
    """1 and 10 steps of decaying isotropic turbulence: rel L2 of u < 1e-10."""
    p = gpu_lib.workload_params("iso_decay", n)
    o, s = _pair(gpu_lib, p)
    t = 0.0
    for step in range(1, 11):
        t, dt = o.step(step, t)
        dtg = s.step(step)
        assert dtg == pytest.approx(dt, rel=0, abs=0)
        if step in (1, 10):
            e = rel_l2_fields(s.get_state(), o.get_state())
            assert e < 1e-10, (step, e)
    assert s.simtime == pytest.approx(t, rel=1e-15)
    div = divergence(p, s.get_state())
    umax = max(np.abs(c).max() for c in s.get_state())
    assert np.abs(div).max() < 1e-13 * max(umax, 1.0) * (n / 3)
    # RK registers match too
    assert rel_l2_fields(s.get_rk(), o.get_rk()) < 1e-10
    s.close()


def test_stats_parity_100_steps(gpu_lib):
    """E(k) and epsilon within 1e-8 over 100 steps (32^3 decaying turbulence)."""
    p = gpu_lib.workload_params("iso_decay", 32)
    o, s = _pair(gpu_lib, p)
    t = 0.0
    worst_e, worst_eps = 0.0, 0.0
    for step in range(1, 101):
        ek_g, tke_g, eps_g, _ = s.stats()
        ek_o, tke_o, eps_o = o.stats()
        worst_e = max(worst_e, rel_l2(ek_g, ek_o))
        worst_eps = max(worst_eps, abs(eps_g - eps_o) / abs(eps_o))
        assert tke_g == pytest.approx(tke_o, rel=1e-8)
        t, _ = o.step(step, t)
        s.step(step)
    # the statistics recorded inside the step (stage 1) are those of the state at step start
    ek_l, tke_l, eps_l, ucfl_l = s.stats(last_step=True)
    s.close()
    assert worst_e < 1e-8 and worst_eps < 1e-8, (worst_e, worst_eps)
    assert ucfl_l > 0


def test_forced_parity(gpu_lib):
    """Forced isotropic turbulence: OU forcing coefficients and u after 10 steps."""
    p = gpu_lib.workload_params("iso_forced_particles", 32)
    p.p_track_part = 0
    o, s = _pair(gpu_lib, p)
    t = 0.0
    for step in range(1, 11):
        t, _ = o.step(step, t)
        s.step(step)
        if step in (1, 10):
            assert rel_l2_fields(s.get_forcing(), o.get_forcing()) < 1e-13, step
            assert rel_l2_fields(s.get_state(), o.get_state()) < 1e-10, step
    s.close()


def test_forced_parity_wide_band(gpu_lib):
    """Forcing radius 6.5 (3315 normal pairs per stage, 61 KB of shared memory in the
    stage-scalar kernel, above the 48 KB launch default): forcing and u after 3 steps."""
    p = gpu_lib.workload_params("iso_forced_particles", 32)
    p.p_track_part = 0
    p.force_kf = 6.5
    p.force_sigma = 0.01
    o, s = _pair(gpu_lib, p)
    t = 0.0
    for step in range(1, 4):
        t, _ = o.step(step, t)
        s.step(step)
    assert rel_l2_fields(s.get_forcing(), o.get_forcing()) < 1e-13
    assert rel_l2_fields(s.get_state(), o.get_state()) < 1e-10
    s.close()


def test_particle_parity(gpu_lib):
    """Tracers: positions within 1e-10 after 10 steps (same initial positions)."""
    p = gpu_lib.workload_params("iso_forced_particles", 32)
    p.p_np_global = 4096
    o, s = _pair(gpu_lib, p)
    s.init_particles()
    xp, up, ur, pr, dp = s.get_particles()
    o.set_particles(xp, up, ur, pr, dp)
    t = 0.0
    for step in range(1, 11):
        t, _ = o.step(step, t)
        s.step(step)
        if step in (1, 10):
            xg = s.get_particles()[0]
            xo = o.get_particles(p.p_np_global)[0]
            d = np.abs(xg - xo)
            d = np.minimum(d, 2 * np.pi - d)      # a wrap on one side only is not an error
            assert d.max() < 1e-10, (step, d.max())
    # physical velocity materialised for the particles matches the oracle's
    assert rel_l2_fields(s.physical_velocity(), o.get_physical()) < 1e-12
    s.check_status()
    s.close()


def test_particle_init_matches_oracle(gpu_lib):
    import oracle as O
    p = gpu_lib.workload_params("iso_forced_particles", 32)
    p.p_np_global = 10000
    o = O.Oracle(p)
    o.init_particles()
    with gpu_lib.Simulation(p) as s:
        s.init_particles()
        xg = s.get_particles()[0]
    xo = o.get_particles(p.p_np_global)[0]
    assert np.abs(xg - xo).max() < 1e-14
    dx = 2 * np.pi / 32
    assert xg.min() >= -dx / 2 and xg.max() < 2 * np.pi - dx / 2


@pytest.mark.parametrize("order", [1, 2, 3, 5, 6])
def test_particle_parity_orders(gpu_lib, order):
    """Interpolation orders other than 4 (p_InterpInterpolate3D takes 1..6), 1001 tracers
    (a partial thread group and a partial CTA at the tail): positions after 3 steps."""
    p = gpu_lib.workload_params("iso_forced_particles", 32)
    p.p_np_global = 1001
    p.p_interp_order = order
    o, s = _pair(gpu_lib, p)
    s.init_particles()
    xp, up, ur, pr, dp = s.get_particles()
    o.set_particles(xp, up, ur, pr, dp)
    t = 0.0
    for step in range(1, 4):
        t, _ = o.step(step, t)
        s.step(step)
    xg = s.get_particles()[0]
    xo = o.get_particles(p.p_np_global)[0]
    d = np.abs(xg - xo)
    d = np.minimum(d, 2 * np.pi - d)
    assert d.max() < 1e-10, d.max()
    s.check_status()
    s.close()


def test_inertial_particles(gpu_lib):
    p = gpu_lib.workload_params("iso_forced_particles", 32)
    p.p_np_global = 1024
    p.p_dia_vals = 0.01
    p.p_rho = 1000.0
    o, s = _pair(gpu_lib, p)
    s.init_particles()
    o.set_particles(*s.get_particles())
    t = 0.0
    for step in range(1, 6):
        t, _ = o.step(step, t)
        s.step(step)
    xg, ug = s.get_particles()[:2]
    xo, uo = o.get_particles(p.p_np_global)[:2]
    s.close()
    assert rel_l2(ug, uo) < 1e-10
    d = np.abs(xg - xo)
    assert np.minimum(d, 2 * np.pi - d).max() < 1e-10


def test_stage_api_matches_step(gpu_lib):
    """f_RK3Stage1..3 called one by one equals g_RK3Calc."""
    p = gpu_lib.workload_params("iso_decay", 32)
    a = gpu_lib.Simulation(p)
    b = gpu_lib.Simulation(p)
    a.init_fluid()
    b.init_fluid()
    a.step(1)
    dt = 0.0
    dt = gpu_lib.f_RK3Stage1(1, 0.0, dt, sim=b)
    dt = gpu_lib.f_RK3Stage2(1, dt / 3, dt, sim=b)
    dt = gpu_lib.f_RK3Stage3(1, 0.75 * dt, dt, sim=b)
    e = rel_l2_fields(a.get_state(), b.get_state())
    a.close()
    b.close()
    assert e < 1e-15


def test_advance_matches_steps(gpu_lib):
    p = gpu_lib.workload_params("iso_forced_particles", 32)
    p.p_np_global = 512
    a = gpu_lib.Simulation(p)
    b = gpu_lib.Simulation(p)
    for s in (a, b):
        s.init_fluid()
        s.init_particles()
    for _ in range(5):
        a.step()
    b.advance(5)
    assert b.simtime == pytest.approx(a.simtime, rel=1e-15)
    assert rel_l2_fields(a.get_state(), b.get_state()) < 1e-15
    assert np.array_equal(a.get_particles()[0], b.get_particles()[0])
    a.close()
    b.close()


def test_nan_detection(gpu_lib):
    p = gpu_lib.workload_params("iso_decay", 16)
    with gpu_lib.Simulation(p) as s:
        s.init_fluid()
        u = s.get_state()
        u[0][1, 1, 1] = np.nan
        s.set_state(u)
        with pytest.raises(gpu_lib.PandoraError) as ei:
            s.check_status()
        assert ei.value.status == -4
        s.init_fluid()
        s.check_status()   # status word was cleared and the state is finite again


def test_pass_timing_instrumentation(gpu_lib):
    """Event pairs around every pass: durations for all 3 stages x 6 passes, and the
    instrumented step computes exactly what the plain step does."""
    p = gpu_lib.workload_params("iso_forced_particles", 32)
    p.p_np_global = 512
    a = gpu_lib.Simulation(p)
    b = gpu_lib.Simulation(p)
    for s in (a, b):
        s.init_fluid()
        s.init_particles()
    b.set_pass_timing(0x3F)
    for step in range(1, 3):
        a.step(step)
        b.step(step)
    t = b.pass_times()
    assert t.shape == (3, 6) and (t > 0).all(), t
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)
    assert np.array_equal(a.get_particles()[0], b.get_particles()[0])
    b.set_pass_timing(1 << 2)          # the x pass only
    b.step(3)
    t = b.pass_times()
    assert (t[:, 2] > 0).all() and (np.delete(t, 2, axis=1) == -1).all(), t
    b.set_pass_timing(0)
    b.step(4)
    assert (b.pass_times() == -1).all()
    a.close()
    b.close()


def test_run_module(gpu_lib):
    """The profiling driver `python -m pandora.run` on a small anisotropic case."""
    from pandora import run
    assert run.main(["--workload", "shear", "--nodes", "64", "32", "48", "--steps", "2"]) == 0
    assert run.main(["--workload", "iso_forced_particles", "--nodes", "32", "32", "32", "--steps", "1",
                     "--np", "256", "--precision", "fp32_mixed"]) == 0
    assert run.main(["--workload", "iso_decay", "--nodes", "32", "32", "32", "--steps", "2", "--batch", "4"]) == 0


@pytest.mark.parametrize("mode,cut", [(2, 1.0), (3, 0.7)])
def test_dealias_parity(gpu_lib, mode, cut):
    """DEALIASING 2 (2/3 sphere) and 3 (LES cutoff): truncated initial field, then
    10 steps with the truncation at every stage's start (src/pf_rk3.f90:269-277)."""
    import oracle as O
    p = gpu_lib.workload_params("iso_decay", 32)
    p.dealiasing, p.les_cutoff = mode, cut
    o = O.Oracle(p)
    o.init_fluid()
    with gpu_lib.Simulation(p) as s:
        s.init_fluid()
        assert rel_l2_fields(s.get_state(), o.get_state()) < 1e-13
        t = 0.0
        for step in range(1, 11):
            t, _ = o.step(step, t)
            s.step(step)
        assert rel_l2_fields(s.get_state(), o.get_state()) < 1e-10
        ek_g, tke_g, eps_g, _ = s.stats()
        ek_o, tke_o, eps_o = o.stats()
        assert rel_l2(ek_g, ek_o) < 1e-8 and abs(eps_g - eps_o) < 1e-8 * abs(eps_o)
        assert rel_l2_fields(s.nonlinear(), o.nonlinear()) < 1e-12


@pytest.mark.parametrize("workload", ["iso_decay", "shear", "shear_rconv"])
def test_realspace_stats_parity(gpu_lib, workload):
    """Real-space moments and maxima (f_FluidstatsRs2D) of the same state on both sides;
    in the R-conv form the "vorticity" moments are those of d(u1,u2,u3)/dx1, the fields
    the reference holds in u4..u6 there."""
    import oracle as O
    p = gpu_lib.workload_params("shear" if workload == "shear_rconv" else workload, 32)
    p.p_track_part = 0
    if workload == "shear_rconv":
        p.ns_deformed = gpu_lib.NS_R_CONV
    o, s = _pair(gpu_lib, p)
    t = 0.0
    for step in range(1, 4):
        t, _ = o.step(step, t)
        s.step(step)
    g = s.realspace_sums()
    r = o.realspace_sums()
    s.close()
    np.testing.assert_allclose(g[:21], r[:21], rtol=1e-11, atol=1e-12 * np.abs(r[:21]).max())
    np.testing.assert_allclose(g[21:], r[21:], rtol=1e-12)


def test_particle_stats(gpu_lib):
    p = gpu_lib.workload_params("iso_forced_particles", 32)
    p.p_np_global = 1000
    p.p_dia_vals, p.p_rho = 0.01, 1000.0   # inertial: dp > 0, so the kinetic-energy sum is not zero
    with gpu_lib.Simulation(p) as s:
        s.init_fluid()
        s.init_particles()
        s.advance(3)
        d = s.particle_stats()
        _, up, _, _, dp = s.get_particles()
    n = 1000.0
    assert d["u1u1"] == pytest.approx((up[:, 0] ** 2).sum() / n, rel=1e-12)
    assert d["u2u3"] == pytest.approx((up[:, 1] * up[:, 2]).sum() / n, rel=1e-12, abs=1e-15)
    pken = (0.5 * (np.pi / 6.0) * dp ** 3 * 1000.0 * (up ** 2).sum(axis=1)).sum() / n
    assert pken > 0.0 and d["pken"] == pytest.approx(pken, rel=1e-12)


@pytest.mark.parametrize("case", ["iso", "aniso", "shear", "shear_sphere", "fp32"])
def test_x_correlation_parity(gpu_lib, case):
    """TS_CORR's lag sums (src/pf_fluidstats.f90:933-945): the GPU's co-spectrum form
    against the oracle's lag loop on the same state, after a few steps (shear: a frame with
    binv(1,3) != 0; shear_sphere: DEALIASING 2, the dropped modes left out)."""
    import oracle as O
    wl = "shear" if case.startswith("shear") else "iso_decay"
    p = gpu_lib.workload_params(wl, 32)
    p.p_track_part = 0
    if case == "aniso":
        p.nodes_x, p.nodes_y, p.nodes_z = 48, 32, 24
    if case == "shear_sphere":
        p.dealiasing = 2
    if case == "fp32":
        p.precision = gpu_lib.PREC_FP32_MIXED
    s = gpu_lib.Simulation(p)
    s.init_fluid()
    s.advance(3)
    q = p.copy()
    q.precision = gpu_lib.PREC_FP64
    o = O.Oracle(q)
    o.set_state(s.get_state())
    if wl == "shear":
        o.update_b(4, s.simtime)
        assert o.frame() == pytest.approx(s.frame(), rel=1e-14)
    g = s.x_correlation_sums()
    want = o.x_correlation()[:-1]
    tol = 1e-5 if case == "fp32" else 1e-12
    assert np.abs(g - want).max() < tol * abs(want[0]), np.abs(g - want).max() / abs(want[0])
    d = s.realspace_stats(corr=True)
    assert d["r1i"].size == p.nodes_x // 2 + 1 and d["lint11"] != 0.0
    if wl != "shear":    # lag 0 is u1u1 itself (for shear a product of laboratory and stored u1)
        assert d["r1i"][0] == pytest.approx(1.0, rel=1e-6 if case == "fp32" else 1e-12)
    s.close()



@pytest.mark.parametrize("workload,n", [("iso_decay", 64), ("iso_forced_particles", 32)])
def test_integrating_factor_parity(gpu_lib, workload, n):
    """PANDORA_VISCOUS_INTEGRATING_FACTOR against the oracle's same mode: u, the RK
    register and (forced case) the tracers after 1 and 10 steps; the explicit form of the
    same run differs from it by the scheme's O(dt^3) local error, not by round-off."""
    p = gpu_lib.workload_params(workload, n)
    p.rk3_viscous = gpu_lib.VISCOUS_INTEGRATING_FACTOR
    if p.p_track_part:
        p.p_np_global = 2048
    o, s = _pair(gpu_lib, p, init="gpu")
    if p.p_track_part:
        s.init_particles()
        o.set_particles(*s.get_particles())
    q = p.copy()
    q.rk3_viscous = gpu_lib.VISCOUS_EXPLICIT
    with gpu_lib.Simulation(q) as x:
        x.set_state(s.get_state())
        if p.p_track_part:
            x.set_particles(*s.get_particles())
        t = 0.0
        for step in range(1, 11):
            t, dt = o.step(step, t)
            assert s.step(step) == dt
            x.step(step)
            if step in (1, 10):
                assert rel_l2_fields(s.get_state(), o.get_state()) < 1e-10, step
                assert rel_l2_fields(s.get_rk(), o.get_rk()) < 1e-10, step
        dev = rel_l2_fields(x.get_state(), s.get_state())
    assert 1e-12 < dev < 1e-4, dev
    if p.p_track_part:
        xg = s.get_particles()[0]
        xo = o.get_particles(p.p_np_global)[0]
        d = np.abs(xg - xo)
        assert np.minimum(d, 2 * np.pi - d).max() < 1e-10
    s.close()


def test_integrating_factor_mixed_and_shear_refused(gpu_lib):
    """The FP32-mixed form of the integrating factor against the FP64 oracle (1e-5), and
    the sheared flow refused (its wavenumbers move with the frame)."""
    import oracle as O
    p = gpu_lib.workload_params("iso_decay", 32)
    p.rk3_viscous = gpu_lib.VISCOUS_INTEGRATING_FACTOR
    o = O.Oracle(p)
    o.init_fluid()
    q = p.copy()
    q.precision = gpu_lib.PREC_FP32_MIXED
    with gpu_lib.Simulation(q) as s:
        s.set_state(o.get_state())
        t = 0.0
        for step in range(1, 6):
            t, _ = o.step(step, t)
            s.step(step)
        assert rel_l2_fields(s.get_state(), o.get_state()) < 1e-5
    r = gpu_lib.workload_params("shear", 32)
    r.rk3_viscous = gpu_lib.VISCOUS_INTEGRATING_FACTOR
    with pytest.raises(gpu_lib.PandoraError) as ei:
        gpu_lib.Simulation(r)
    assert ei.value.status == -10


@pytest.mark.parametrize("dims,workload", [((80, 80, 80), "iso_forced_particles"), ((112, 160, 224), "iso_decay"),
                                           ((56, 40, 320), "shear")])
def test_step_parity_factor_5_and_7_lengths(gpu_lib, dims, workload):
    """Whole steps on grids with factors 5 and 7: forced flow with tracers, decaying flow on
    an anisotropic grid, BF-rot shear; u (and tracers) against the oracle after 3 steps."""
    p = gpu_lib.workload_params(workload, 32)
    p.nodes_x, p.nodes_y, p.nodes_z = dims
    if p.p_track_part:
        p.p_np_global = 1024
    o, s = _pair(gpu_lib, p, init="gpu")
    if p.p_track_part:
        s.init_particles()
        o.set_particles(*s.get_particles())
    t = 0.0
    for step in (1, 2, 3):
        t, dt = o.step(step, t)
        assert s.step(step) == dt
    assert rel_l2_fields(s.get_state(), o.get_state()) < 1e-10
    ek_g, _, eps_g, _ = s.stats()
    ek_o, _, eps_o = o.stats()
    assert rel_l2(ek_g, ek_o) < 1e-8 and abs(eps_g - eps_o) < 1e-8 * abs(eps_o)
    if p.p_track_part:
        d = np.abs(s.get_particles()[0] - o.get_particles(p.p_np_global)[0])
        assert np.minimum(d, 2 * np.pi - d).max() < 1e-10
    s.close()


@pytest.mark.parametrize("dims,workload", [((16, 16, 16), "iso_forced_particles"), ((24, 32, 16), "iso_decay"),
                                           ((32, 32, 32), "shear"), ((48, 24, 32), "iso_forced_particles"),
                                           ((64, 32, 48), "shear"), ((56, 40, 16), "iso_decay")])
def test_x_lines_per_warp_schedules_agree(gpu_lib, dims, workload):
    """The x pass with 1, 2 or 4 lines per warp (x lengths up to 64) does the same
    arithmetic per line: the states (and tracers) after 3 steps are equal bit for bit,
    and equal the oracle's to 1e-10."""
    p = gpu_lib.workload_params(workload, 32)
    p.nodes_x, p.nodes_y, p.nodes_z = dims
    if p.p_track_part:
        p.p_np_global = 512
    out = []
    for lpw in (1, 2, 4):
        q = p.copy()
        q.x_lines_per_warp = lpw
        with gpu_lib.Simulation(q) as s:
            s.init_fluid()
            if q.p_track_part:
                s.init_particles()
            s.advance(3)
            out.append((s.get_state(), s.get_particles()[0] if q.p_track_part else None, s.stats()))
    for u, xp, st in out[1:]:
        assert all(np.array_equal(a, b) for a, b in zip(u, out[0][0]))
        if xp is not None:
            assert np.array_equal(xp, out[0][1])
        assert st[1] == pytest.approx(out[0][2][1], rel=1e-13)
    import oracle as O
    o = O.Oracle(p)
    with gpu_lib.Simulation(p) as s:
        s.init_fluid()
        o.set_state(s.get_state())
        if p.p_track_part:
            s.init_particles()
            o.set_particles(*s.get_particles())
    t = 0.0
    for step in (1, 2, 3):
        t, _ = o.step(step, t)
    assert rel_l2_fields(out[2][0], o.get_state()) < 1e-10
    if p.p_track_part:
        d = np.abs(out[2][1] - o.get_particles(p.p_np_global)[0])
        assert np.minimum(d, 2 * np.pi - d).max() < 1e-10


def test_x_lines_per_warp_validation(gpu_lib):
    p = gpu_lib.workload_params("iso_decay", 32)
    p.x_lines_per_warp = 3
    with pytest.raises(gpu_lib.PandoraError):
        gpu_lib.Simulation(p)
    p = gpu_lib.workload_params("iso_decay", 96)
    p.x_lines_per_warp = 2
    with pytest.raises(gpu_lib.PandoraError):
        gpu_lib.Simulation(p)


def test_particle_count_limit(gpu_lib):
    """More tracers than the per-step sort's 32-bit offsets can count is refused at create,
    before any allocation."""
    p = gpu_lib.workload_params("iso_forced_particles", 32)
    p.p_np_global = 1 << 31
    with pytest.raises(gpu_lib.PandoraError):
        gpu_lib.Simulation(p)
