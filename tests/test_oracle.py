"""The CPU oracle against the reference's known-answer test, the committed
fixtures, numpy.fft and the invariants of the discretisation (no GPU)."""
import json
import os

import numpy as np
import pytest

from helpers import divergence, rel_l2_fields, wavenumbers

HERE = os.path.dirname(os.path.abspath(__file__))


def _o(p):
    import oracle as O
    return O.Oracle(p)


@pytest.mark.parametrize("n", [2, 3, 5, 7, 12, 16, 24, 48, 96, 128, 192, 256, 512, 1024])
def test_fft_matches_numpy(n):
    import oracle as O
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    np.testing.assert_allclose(O.fft(x, -1), np.fft.fft(x), rtol=0, atol=1e-13 * np.abs(x).sum())
    np.testing.assert_allclose(O.fft(x, +1), np.fft.ifft(x) * n, rtol=0, atol=1e-13 * np.abs(x).sum())


@pytest.mark.parametrize("n", [32, 48, 64])
def test_nonlinear_known_answer(n):
    """src/ptf_rk3.f90:1179-1181 -- the reference's own expected L1 norms."""
    from pandora.params import default_params
    kat = json.load(open(os.path.join(HERE, "golden", "kat_nonlinear.json")))
    p = default_params(n)
    o = _o(p)
    o.init_taylor_green_reverse()
    u = o.get_state()
    nkj, nkk = o.nkj, o.nkk
    for m in kat["modes"]:
        j = m["j"] % nkj
        k = m["k"] % nkk
        for c in range(3):
            assert u[c][m["i"], j, k] == m["u"][c]
    nl = o.nonlinear()
    l1 = [float(np.abs(c.real).sum() + np.abs(c.imag).sum()) for c in nl]
    np.testing.assert_allclose(l1, kat["l1_norms"], rtol=1e-13)


def test_transform_round_trip_and_physical_values():
    """spectral -> physical is FFTW BACKWARD (unnormalised): a single mode
    u1(i=1,j=0,k=0) = a gives u1(x) = 2 Re(a e^{ix}); the NL of any field maps
    back consistently."""
    from pandora.params import default_params
    p = default_params(16)
    p.f_nu = 0.0
    o = _o(p)
    u = [np.zeros(o.shape, complex) for _ in range(3)]
    a = 0.3 - 0.2j
    u[1][1, 0, 0] = a
    o.set_state(u)
    o.nonlinear()   # fills the physical arrays as a by-product
    phys = o.get_physical()
    x = np.arange(16) * 2 * np.pi / 16
    expect = 2 * (a * np.exp(1j * x)).real
    np.testing.assert_allclose(phys[1][0, 0, :], expect, atol=1e-15)
    np.testing.assert_allclose(phys[1][5, 7, :], expect, atol=1e-15)
    assert np.abs(phys[0]).max() == 0 and np.abs(phys[2]).max() == 0


def test_nonlinear_conserves_energy():
    """The projected, dealiased nonlinear term transfers but does not create
    energy: sum_k w_k Re(u* . P NL) = 0 (w = 2 off the i=0 plane)."""
    from pandora.params import workload_params
    p = workload_params("iso_decay", 32)
    o = _o(p)
    o.init_fluid()
    u = o.get_state()
    nl = o.nonlinear()
    k1, k2, k3 = wavenumbers(p)
    kk = k1 ** 2 + k2 ** 2 + k3 ** 2
    kk[0, 0, 0] = 1
    kdn = k1 * nl[0] + k2 * nl[1] + k3 * nl[2]
    pn = [nl[0] - k1 * kdn / kk, nl[1] - k2 * kdn / kk, nl[2] - k3 * kdn / kk]
    w = np.full(o.shape, 2.0)
    w[0] = 1.0
    tr = sum(np.sum(w * (np.conj(u[c]) * pn[c]).real) for c in range(3))
    scale = sum(np.sum(w * np.abs(u[c]) * np.abs(pn[c])) for c in range(3))
    assert abs(tr) < 1e-13 * scale


def test_single_mode_viscous_decay_is_rk3_polynomial():
    """A single real mode has omega x u = grad(...) which the projection removes,
    so one step multiplies it by 1 + z + z^2/2 + z^3/6, z = -nu k^2 dt (the
    Williamson low-storage scheme is third order on linear problems)."""
    from pandora.params import default_params, RK3_TIMESTEP_FIXED
    p = default_params(16)
    p.f_nu, p.rk3_timestep, p.rk3_dt, p.force_stop = 0.05, RK3_TIMESTEP_FIXED, 0.01, 0
    o = _o(p)
    u = [np.zeros(o.shape, complex) for _ in range(3)]
    u[1][2, 0, 1] = 0.5 + 0.1j      # k = (2, 0, 1), u along y: solenoidal
    o.set_state(u)
    o.step(1, 0.0)
    z = -p.f_nu * 5 * p.rk3_dt
    g = 1 + z + z * z / 2 + z ** 3 / 6
    v = o.get_state()
    assert abs(v[1][2, 0, 1] - (0.5 + 0.1j) * g) < 1e-15
    assert max(np.abs(c).max() for c in (v[0], v[2])) < 1e-17


def test_integrating_factor_single_mode_decays_exactly():
    """The integrating-factor form integrates the viscous term exactly: a single mode
    (whose projected nonlinear term is zero) decays by exp(-nu k^2 dt) per step, for any
    dt, where the explicit form gives the RK3 polynomial."""
    from pandora.params import default_params, RK3_TIMESTEP_FIXED, VISCOUS_INTEGRATING_FACTOR
    for dt in (0.01, 0.5):
        p = default_params(16)
        p.f_nu, p.rk3_timestep, p.rk3_dt, p.force_stop = 0.05, RK3_TIMESTEP_FIXED, dt, 0
        p.rk3_viscous = VISCOUS_INTEGRATING_FACTOR
        o = _o(p)
        u = [np.zeros(o.shape, complex) for _ in range(3)]
        u[1][2, 0, 1] = 0.5 + 0.1j
        o.set_state(u)
        t = 0.0
        for s in (1, 2):
            t, _ = o.step(s, t)
        want = (0.5 + 0.1j) * np.exp(-p.f_nu * 5 * 2 * dt)
        v = o.get_state()
        assert abs(v[1][2, 0, 1] - want) < 2e-16, dt
        assert max(np.abs(c).max() for c in (v[0], v[2])) < 1e-17


def test_integrating_factor_agrees_with_explicit_to_third_order():
    """Both forms are third order in dt: on the same turbulent field over the same time,
    halving dt divides their difference by about 8."""
    from pandora.params import workload_params, VISCOUS_INTEGRATING_FACTOR
    diffs = []
    for dt, nsteps in ((0.01, 4), (0.005, 8)):
        out = []
        for visc in (0, VISCOUS_INTEGRATING_FACTOR):
            p = workload_params("iso_decay", 16)
            p.rk3_dt, p.rk3_viscous = dt, visc
            o = _o(p)
            o.init_fluid()
            t = 0.0
            for s in range(1, nsteps + 1):
                t, _ = o.step(s, t)
            out.append(o.get_state())
            assert np.abs(divergence(p, out[-1])).max() < 1e-16
        diffs.append(rel_l2_fields(out[1], out[0]))
    assert 0 < diffs[1] < diffs[0] < 1e-5
    assert 6.0 < diffs[0] / diffs[1] < 10.0, diffs


def test_integrating_factor_isotropic_only():
    from pandora.params import workload_params, VISCOUS_INTEGRATING_FACTOR
    p = workload_params("shear", 16)
    p.p_track_part = 0
    p.rk3_viscous = VISCOUS_INTEGRATING_FACTOR
    o = _o(p)
    o.init_fluid()
    with pytest.raises(RuntimeError):
        o.step(1, 0.0)


def test_step_invariants_and_fixture_decay():
    from pandora.params import workload_params
    g = np.load(os.path.join(HERE, "golden", "iso_decay_16_3.npz"))
    p = workload_params("iso_decay", 16)
    p.p_track_part = 0
    o = _o(p)
    o.init_fluid()
    assert rel_l2_fields(o.get_state(), list(g["u0"])) < 1e-15
    t = 0.0
    for s in range(1, 4):
        t, _ = o.step(s, t)
    assert rel_l2_fields(o.get_state(), list(g["u"])) < 1e-14
    assert rel_l2_fields(o.get_rk(), list(g["rk"])) < 1e-14
    ek, tke, eps = o.stats()
    np.testing.assert_allclose(ek, g["ek"], rtol=1e-13)
    assert tke == pytest.approx(float(g["tke"]), rel=1e-13)
    assert eps == pytest.approx(float(g["eps"]), rel=1e-13)
    assert np.abs(divergence(p, o.get_state())).max() < 1e-16


def test_fixture_forced_particles():
    from pandora.params import workload_params
    g = np.load(os.path.join(HERE, "golden", "iso_forced_particles_24_3.npz"))
    p = workload_params("iso_forced_particles", 24)
    p.p_np_global = 64
    o = _o(p)
    o.init_fluid()
    o.init_particles()
    np.testing.assert_array_equal(o.get_particles(64)[0], g["x0"])
    t = 0.0
    for s in range(1, 4):
        t, _ = o.step(s, t)
    assert rel_l2_fields(o.get_state(), list(g["u"])) < 1e-14
    assert rel_l2_fields(o.get_forcing(), list(g["forcing"])) < 1e-14
    np.testing.assert_allclose(o.get_particles(64)[0], g["x"], atol=1e-13)


def test_forcing_draw_count_and_symmetry():
    from pandora.params import workload_params
    p = workload_params("iso_forced_particles", 16)
    p.p_track_part = 0
    o = _o(p)
    assert o.force_calls_per_stage() == 195   # NK = 2: 3*(9 + 6) + 3*2*25
    o.init_fluid()
    o.step(1, 0.0)
    f = o.get_forcing()
    nk = 2
    for c in f:
        pl = c[0]        # i = 0 plane, index [j+NK][k+NK]
        for j in range(-nk, nk + 1):
            for k in range(-nk, nk + 1):
                if (j, k) == (0, 0):
                    continue
                assert pl[j + nk, k + nk] == np.conj(pl[-j + nk, -k + nk])


def test_forcing_stops():
    from pandora.params import workload_params
    p = workload_params("iso_forced_particles", 16)
    p.p_track_part = 0
    p.force_stop = 2
    o = _o(p)
    o.init_fluid()
    o.step(1, 0.0)
    assert max(np.abs(c).max() for c in o.get_forcing()) > 0
    o.step(2, 0.0)
    assert max(np.abs(c).max() for c in o.get_forcing()) == 0


def test_interpolation_order_four():
    """4-point Lagrange (Neville) reproduces node values and converges at 4th
    order on a smooth periodic field."""
    from pandora.params import default_params
    errs = []
    for n in (16, 32):
        p = default_params(n)
        p.p_track_part = 1
        p.p_interp_order = 4
        o = _o(p)
        u = [np.zeros(o.shape, complex) for _ in range(3)]
        u[0][1, 0, 0] = 0.5          # u1 = cos(x)
        u[0][0, 1, 0] = 0.25         # + 0.5 cos(y): the i=0 plane holds both
        u[0][0, -1, 0] = 0.25        #   conjugate partners
        o.set_state(u)
        o.nonlinear()
        rng = np.random.default_rng(1)
        dx = 2 * np.pi / n
        xp = rng.uniform(-dx / 2, 2 * np.pi - dx / 2, size=(200, 3))
        uf = o.interpolate(xp)
        exact = np.cos(xp[:, 0]) + 0.5 * np.cos(xp[:, 1])
        errs.append(np.abs(uf[:, 0] - exact).max())
        nodes = np.stack([np.arange(5) * dx, np.arange(5) * dx, np.zeros(5)], axis=1)
        np.testing.assert_allclose(o.interpolate(nodes)[:, 0], np.cos(nodes[:, 0]) + 0.5 * np.cos(nodes[:, 1]),
                                   atol=1e-15)
    assert errs[0] / errs[1] > 12   # ~16 for 4th order


def test_particle_wrap_asymmetry():
    """x3 wraps with '>' where x1, x2 wrap with '>=' (src/pp_mpi.f90:1011-1057)."""
    from pandora.params import default_params
    p = default_params(16)
    p.p_track_part, p.p_ts_release, p.f_nu = 1, 1, 0.0
    p.rk3_timestep, p.rk3_dt = 2, 0.01
    o = _o(p)
    dx = 2 * np.pi / 16
    lo = -dx / 2
    xp = np.array([[lo - 1e-3, 1.0, 1.0], [1.0, 2 * np.pi + lo + 1e-3, 1.0]])
    o.set_particles(xp, np.zeros_like(xp), np.zeros_like(xp), np.zeros_like(xp), np.zeros(2))
    o.step(1, 0.0)
    x = o.get_particles(2)[0]
    assert lo <= x[0, 0] < 2 * np.pi + lo
    assert lo <= x[1, 1] < 2 * np.pi + lo


def test_stats_shells():
    from pandora.params import workload_params
    p = workload_params("iso_decay", 32)
    o = _o(p)
    o.init_fluid()
    ek, tke, eps = o.stats()
    assert len(ek) == round((3 * 10 ** 2) ** 0.5)
    assert tke > 0 and eps > 0
    # spectrum peaks near kp = 4
    assert 3 <= int(np.argmax(ek)) + 1 <= 5


@pytest.mark.parametrize("mode,cut", [(2, 1.0), (3, 0.6)])
def test_dealias_spherical_and_les(mode, cut):
    """src/pf_arrays.f90:1865-1987: DEALIASING 2 keeps |k| <= KMAX, 3 keeps
    |k| <= LES_CUTOFF * KMAX; the initial field and every stage's state are truncated."""
    from pandora.params import workload_params
    p = workload_params("iso_decay", 32)
    p.dealiasing, p.les_cutoff = mode, cut
    o = _o(p)
    o.init_fluid()
    k1, k2, k3 = wavenumbers(p)
    km = np.sqrt(k1 ** 2 + k2 ** 2 + k3 ** 2)
    kmax = cut * (32 // 3)
    out = km > kmax
    u = o.get_state()
    assert all(np.abs(c[out]).max() == 0.0 for c in u)
    assert all(np.abs(c[~out]).max() > 0.0 for c in u)
    t = 0.0
    for step in range(1, 3):
        t, _ = o.step(step, t)
    # after a step the update has refilled the corners; the next stage truncates again
    u = o.get_state()
    assert max(np.abs(c[out]).max() for c in u) > 0.0
    o.nonlinear()
    u = o.get_state()
    assert all(np.abs(c[out]).max() == 0.0 for c in u)
    assert np.abs(divergence(p, u)).max() < 1e-13


def test_dealias_default_is_the_two_thirds_cube():
    from pandora.params import workload_params
    p = workload_params("iso_decay", 32)
    assert p.dealiasing == 1
    o = _o(p)
    o.init_fluid()
    k1, k2, k3 = wavenumbers(p)
    out = np.sqrt(k1 ** 2 + k2 ** 2 + k3 ** 2) > 32 // 3
    assert max(np.abs(c[out]).max() for c in o.get_state()) > 0.0


@pytest.mark.parametrize("workload", ["iso_decay", "shear"])
def test_realspace_sums_parseval(workload):
    """f_FluidstatsRs2D's velocity second moments (laboratory frame for shear) carry the
    spectral kinetic energy of f_FluidstatsFs (Parseval)."""
    from pandora.params import workload_params
    from pandora.rk3 import realspace_normalise
    p = workload_params(workload, 32)
    p.p_track_part = 0
    o = _o(p)
    o.init_fluid()
    r = realspace_normalise(o.realspace_sums(), p)
    _, tke, _ = o.stats()
    assert 0.5 * (r["u1u1"] + r["u2u2"] + r["u3u3"]) == pytest.approx(tke, rel=1e-12)
    assert 2.0 < r["flat1"] < 4.5 and abs(r["skew2"]) < 1.0



def _cospectrum_correlation(p, u, bi13):
    """r[l] = N^3 sum_m c_m Re(P_m e^{-2 pi i m l / NX}) with P_m = sum_{j,k} a conj(b),
    a = u1 in the laboratory frame, b = the stored u1: the wave-space form of the lag sums."""
    b = u[0]
    a = b if p.f_type == 1 else float(p.b110) * u[0] + bi13 * u[2]
    P = np.sum(a * np.conj(b), axis=(1, 2))
    m = np.arange(P.size)
    c = np.where(m == 0, 1.0, 2.0)
    lags = np.arange(p.nodes_x // 2 + 1)
    ph = np.exp(-2j * np.pi * np.outer(lags, m) / p.nodes_x)
    return float(p.nodes_x * p.nodes_y * p.nodes_z) * np.real(ph @ (c * P))


@pytest.mark.parametrize("workload,dims", [("iso_decay", (32, 32, 32)), ("iso_decay", (48, 32, 24)),
                                           ("shear", (32, 32, 32))])
def test_x_correlation_lag_loop_and_cospectrum(workload, dims):
    """TS_CORR (src/pf_fluidstats.f90:933-945): the oracle's lag loop, as the reference runs
    it, equals the co-spectrum form the GPU evaluates; lag 0 is the u1 second moment
    (exactly, for isotropic flow) and lint11 is the lags' sum times dx_laboratoryframe."""
    from pandora.params import workload_params
    from pandora.rk3 import correlation_normalise, realspace_normalise
    p = workload_params(workload, dims[0])
    p.nodes_x, p.nodes_y, p.nodes_z = dims
    p.p_track_part = 0
    o = _o(p)
    o.init_fluid()
    if workload == "shear":
        o.update_b(5, 0.3)            # a frame with binv(1,3) != 0
    out = o.x_correlation()
    r, lint = out[:-1], out[-1]
    want = _cospectrum_correlation(p, o.get_state(), o.frame()[1])
    assert np.abs(r - want).max() < 1e-12 * abs(r[0])
    rs = realspace_normalise(o.realspace_sums(), p)
    if workload == "iso_decay":
        assert r[0] == o.realspace_sums()[0]
    cn = correlation_normalise(r, rs["u1u1"], p)
    assert cn["lint11"] == pytest.approx(lint / (rs["u1u1"] * np.prod(dims)), rel=1e-12)
    if workload == "iso_decay":
        assert cn["r1i"][0] == pytest.approx(1.0, rel=1e-14)
        assert np.all(np.abs(cn["r1i"]) <= 1.0 + 1e-12)
