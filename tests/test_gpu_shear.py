"""Homogeneous shear (Rogallo moving frame, BF-rot formulation) on the GPU
against the oracle, through the C-ABI: state, statistics in the laboratory
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
def test_rogallo_with_particles_unsupported(gpu_lib, form):
    p = _shear(gpu_lib, 32, remesh_t=5, npart=256)
    p.ns_deformed = form
    with pytest.raises(gpu_lib.PandoraError):
        gpu_lib.Simulation(p)


def test_rconv_single_simulations_only(gpu_lib):
    """R-conv has no batched x pass: a batch of R-conv members is refused."""
    p = _shear(gpu_lib, 32, remesh_t=5)
    p.ns_deformed = gpu_lib.NS_R_CONV
    with pytest.raises(gpu_lib.PandoraError):
        gpu_lib.Batch(p, 2)


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
