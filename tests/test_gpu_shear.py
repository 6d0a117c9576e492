"""Homogeneous shear (Rogallo moving frame: the BF-rot, R-rot and R-conv forms) on the
GPU against the oracle, through the C-ABI: state, statistics in the laboratory
frame, frame tensors and particles, across a remesh."""
import numpy as np
import pytest

from helpers import divergence, rel_l2, rel_l2_fields

pytestmark = pytest.mark.gpu


def _shear(pandora, n=32, remesh_t=5, npart=0):
    p = pandora.workload_params("shear", n)
    p.f_remesh_t = remesh_t          # remesh at step B110*remesh_t + 1, then every 2*B110*remesh_t
    if npart:
        p.p_np_global = npart
    else:
        p.p_track_part = 0
    return p


def test_deformed_init_matches_oracle(gpu_lib):
    import oracle as O
    p = _shear(gpu_lib, 48)
    o = O.Oracle(p)
    o.init_fluid()
    with gpu_lib.Simulation(p) as s:
        s.init_fluid()
        assert rel_l2_fields(s.get_state(), o.get_state()) < 1e-13


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_shear_steps_across_remesh(gpu_lib, mode):
    """mode: DEALIASING 1 (2/3 cube), 2 (2/3 sphere in the laboratory frame, also
    applied before and after the remesh, src/pf_rk3.f90:3999-4025) or 3 (LES cutoff 0.8)."""
    import oracle as O
    p = _shear(gpu_lib, 32, remesh_t=5)
    p.dealiasing, p.les_cutoff = mode, 0.8
    o = O.Oracle(p)
    s = gpu_lib.Simulation(p)
    s.init_fluid()
    o.set_state(s.get_state())
    t = 0.0
    for step in range(1, 26):
        t, dt = o.step(step, t)
        dtg = s.step(step)
        assert dtg == dt == pytest.approx((0.5 / p.f_deform_s) / p.f_remesh_t, rel=1e-15)
        if step in (1, 10, 11, 12, 25):      # 11: first remesh (B110 * F_REMESH_T + 1)
            e = rel_l2_fields(s.get_state(), o.get_state())
            assert e < 1e-10, (step, e)
            gb, ob = s.frame(), o.frame()
            assert gb == pytest.approx(ob, rel=1e-14, abs=1e-15), (step, gb, ob)
            ek_g, tke_g, eps_g, _ = s.stats()
            ek_o, tke_o, eps_o = o.stats()
            assert rel_l2(ek_g, ek_o) < 1e-8 and abs(eps_g - eps_o) < 1e-8 * abs(eps_o), step
            assert tke_g == pytest.approx(tke_o, rel=1e-10)
    assert np.abs(divergence(p, s.get_state())).max() < 1e-14
    s.close()


@pytest.mark.parametrize("form", [2, 3])
def test_rogallo_steps_across_remesh(gpu_lib, form):
    """NS_DEFORMED = 2 (R-conv) and 3 (R-rot): laboratory velocity components on the
    sheared wavenumber grid, continuity fixed on the moving components; state, frame
    and statistics against the oracle across the first remesh.  R-conv carries u and
    its nine gradients through the inverse passes."""
    import oracle as O
    p = _shear(gpu_lib, 32, remesh_t=5)
    p.ns_deformed = form
    o = O.Oracle(p)
    s = gpu_lib.Simulation(p)
    s.init_fluid()
    o.set_state(s.get_state())
    t = 0.0
    for step in range(1, 15):
        t, dt = o.step(step, t)
        dtg = s.step(step)
        assert dtg == dt
        if step in (1, 10, 11, 14):
            e = rel_l2_fields(s.get_state(), o.get_state())
            assert e < 1e-10, (step, e)
            assert s.frame() == pytest.approx(o.frame(), rel=1e-14, abs=1e-15), step
            ek_g, tke_g, eps_g, _ = s.stats()
            ek_o, tke_o, eps_o = o.stats()
            assert rel_l2(ek_g, ek_o) < 1e-8 and abs(eps_g - eps_o) < 1e-8 * abs(eps_o), step
            assert tke_g == pytest.approx(tke_o, rel=1e-10)
    s.close()


@pytest.mark.parametrize("dims", [(16, 16, 16), (24, 16, 16), (32, 16, 16), (48, 32, 24), (64, 16, 16),
                                  (96, 16, 16), (128, 16, 16), (192, 16, 16), (256, 16, 16),
                                  (384, 16, 16), (512, 16, 16), (768, 16, 16), (1024, 16, 16),
                                  (16, 96, 16), (16, 16, 96)])
def test_rconv_nonlinear_every_length(gpu_lib, dims):
    """The R-conv product (twelve fields through K1/K2, the four-array x pass) at every
    x length, in a frame with bmat(1,3) != 0 (after two steps)."""
    import oracle as O
    p = _shear(gpu_lib, 32, remesh_t=5)
    p.nodes_x, p.nodes_y, p.nodes_z = dims
    p.ns_deformed = gpu_lib.NS_R_CONV
    o = O.Oracle(p)
    s = gpu_lib.Simulation(p)
    s.init_fluid()
    o.set_state(s.get_state())
    t = 0.0
    for step in (1, 2):
        t, _ = o.step(step, t)
        s.step(step)
    assert s.frame()[0] != 0.0
    assert s.frame() == pytest.approx(o.frame(), rel=1e-14)
    o.set_state(s.get_state())      # the product of one state: no drift of the two runs
    e = rel_l2_fields(s.nonlinear(), o.nonlinear())
    s.close()
    assert e < 1e-12, e


@pytest.mark.parametrize("form", [2, 3])
def test_rogallo_particles_across_remesh(gpu_lib, form):
    """Tracers in the R forms (p_RK3SolveParticleR, src/pp_rk3.f90:307-403): the
    laboratory components of the sheared grid interpolated at the moving position, the
    isotropic RK3 arithmetic, and x1 += x3 at the remesh (step 9 here); positions, the
    state and the particle velocities against the oracle after 12 steps."""
    import oracle as O
    p = _shear(gpu_lib, 32, remesh_t=4, npart=2048)
    p.ns_deformed = form
    o = O.Oracle(p)
    s = gpu_lib.Simulation(p)
    s.init_fluid()
    s.init_particles()
    o.set_state(s.get_state())
    o.set_particles(*s.get_particles())
    t = 0.0
    for step in range(1, 13):
        t, _ = o.step(step, t)
        s.step(step)
    assert rel_l2_fields(s.get_state(), o.get_state()) < 1e-10
    xg, ug = s.get_particles()[:2]
    xo, uo = o.get_particles(p.p_np_global)[:2]
    d = np.abs(xg - xo)
    assert np.minimum(d, 2 * np.pi - d).max() < 1e-10
    assert rel_l2(ug, uo) < 1e-10
    # the physical field the particles read is the laboratory velocity of the last stage
    assert rel_l2_fields(s.physical_velocity(), o.get_physical()) < 1e-12
    s.check_status()
    s.close()


def test_rconv_batch_members_equal_alone_runs(gpu_lib):
    """R-conv members in a batch (the batched four-array x pass and nine-field K1/K2),
    one admitted mid-run, with tracers: each equals its run alone bit for bit."""
    p = _shear(gpu_lib, 32, remesh_t=4, npart=256)
    p.ns_deformed = gpu_lib.NS_R_CONV

    def member(seed):
        q = p.copy()
        q.seed_fluid, q.seed_particles = seed, 500 + seed
        return q

    def alone(q, n):
        with gpu_lib.Simulation(q) as s:
            s.init_fluid()
            s.init_particles()
            for k in range(1, n + 1):
                s.step(k)
            return s.get_state(), s.get_particles()[0]

    with gpu_lib.Batch(p, 2) as b:
        s0 = b.admit(member(61))
        b.step(3)
        s1 = b.admit(member(62))
        b.step(8)                       # the first member crosses its remesh at step 9
        b.sync()
        for slot, seed, n in ((s0, 61, 11), (s1, 62, 8)):
            u, xp = alone(member(seed), n)
            assert all(np.array_equal(x, y) for x, y in zip(b.get_state(slot), u)), seed
            assert np.array_equal(b.get_particles(slot)[0], xp), seed


def test_shear_particles(gpu_lib):
    p = _shear(gpu_lib, 32, remesh_t=4, npart=2048)
    import oracle as O
    o = O.Oracle(p)
    s = gpu_lib.Simulation(p)
    s.init_fluid()
    s.init_particles()
    o.set_state(s.get_state())
    o.set_particles(*s.get_particles())
    t = 0.0
    for step in range(1, 13):              # remesh at step 9
        t, _ = o.step(step, t)
        s.step(step)
    xg = s.get_particles()[0]
    xo = o.get_particles(p.p_np_global)[0]
    d = np.abs(xg - xo)
    d = np.minimum(d, 2 * np.pi - d)
    assert d.max() < 1e-10, d.max()
    s.check_status()
    s.close()


@pytest.mark.parametrize("form", [0, 1, 2, 3])
@pytest.mark.parametrize("dims", [(32, 48, 512), (24, 16, 512)])
def test_staged_k1_lengths_and_forms(gpu_lib, form, dims):
    """z lines of 512 points in FP64 take the K1 whose velocity rows arrive by tensor
    copies (one CTA per tile forming every field): isotropic (0), BF-rot (1), R-rot (2) and
    R-conv (3) against the oracle after 3 steps, the last tile of i partial."""
    import oracle as O
    if form == 0:
        p = gpu_lib.workload_params("iso_decay", 32)
    else:
        # dt = (0.5/S)/F_REMESH_T = 0.002: explicit viscosity stays stable at k3 = 170
        p = _shear(gpu_lib, 32, remesh_t=250)
        p.ns_deformed = {1: gpu_lib.NS_BF_ROT, 2: gpu_lib.NS_R_ROT, 3: gpu_lib.NS_R_CONV}[form]
    p.nodes_x, p.nodes_y, p.nodes_z = dims
    o = O.Oracle(p)
    s = gpu_lib.Simulation(p)
    s.init_fluid()
    o.set_state(s.get_state())
    t = 0.0
    for step in (1, 2, 3):
        t, _ = o.step(step, t)
        s.step(step)
    assert rel_l2_fields(s.get_state(), o.get_state()) < 1e-10
    o.set_state(s.get_state())
    assert rel_l2_fields(s.nonlinear(), o.nonlinear()) < 1e-12
    s.check_status()
    s.close()
