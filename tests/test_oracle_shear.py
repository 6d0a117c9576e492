"""The shear (BF-rot) oracle: closed-form frame, remesh schedule and shift,
fixed shear time step, solenoidal state (no GPU)."""
import numpy as np
import pytest

from helpers import divergence, wavenumbers


def _o(n=24, remesh_t=5):
    import oracle as O
    from pandora.params import workload_params
    p = workload_params("shear", n)
    p.f_remesh_t = remesh_t
    p.p_track_part = 0
    return p, O.Oracle(p)


def test_frame_closed_form_and_remesh_schedule():
    p, o = _o()
    b110, frt, S = p.b110, p.f_remesh_t, p.f_deform_s
    assert [t for t in range(1, 60) if o.remesh_due(t)] == [11, 31, 51]
    o.update_b(5, 0.3)
    b13, bi13 = o.frame()
    assert b13 == pytest.approx(-(1.0 / b110) * S * 0.3) and bi13 == pytest.approx(S * 0.3)
    # after the first remesh the local time restarts at -B110/(2S) (src/pg_rk3.f90:330-339)
    o.update_b(12, 1.2)
    b13, bi13 = o.frame()
    assert bi13 == pytest.approx(S * (1.2 - b110 / S))


def test_remesh_shift_and_frame_jump():
    p, o = _o(24, remesh_t=2)
    o.init_fluid()
    t = 0.0
    for step in range(1, 5):
        t, dt = o.step(step, t)
        assert dt == pytest.approx(0.5 / p.f_deform_s / p.f_remesh_t)
    before = o.get_state()
    o.stage(1, 5, dt)                      # step 5 = B110 * F_REMESH_T + 1: remesh first
    b13, bi13 = o.frame()
    assert bi13 == pytest.approx(-p.b110 / 2.0)
    assert b13 == pytest.approx((1.0 / p.b110) * p.b110 / 2.0)
    after = o.get_state()
    assert not np.allclose(before[2], after[2])


def test_shear_state_stays_solenoidal():
    p, o = _o(24)
    o.init_fluid()
    t = 0.0
    for step in range(1, 16):
        t, _ = o.step(step, t)
    assert np.abs(divergence(p, o.get_state())).max() < 1e-15
    ek, tke, eps = o.stats()
    assert np.isfinite(ek).all() and tke > 0 and eps > 0


@pytest.mark.parametrize("form", [2, 3])
def test_rogallo_continuity_across_remesh(form):
    """R-conv (NS_DEFORMED = 2) and R-rot (3) forms: after a stage's update, the moving
    components bmat u of the stored (laboratory) components are solenoidal,
    k . (bmat u) = 0, in the frame of that stage (f_RK3ContinuityFixRRot), also after
    the remesh."""
    import oracle as O
    from pandora.params import workload_params
    p = workload_params("shear", 32)
    p.f_remesh_t, p.p_track_part, p.ns_deformed = 5, 0, form
    o = O.Oracle(p)
    o.init_fluid()
    t = 0.0
    for step in range(1, 12):   # the remesh is step 11
        t, dt = o.step(step, t)
    o.stage(1, 12, dt)          # stage 1 of step 12 in the frame set at the end of step 11
    u = o.get_state()
    b13, _ = o.frame()
    k1, k2, k3 = wavenumbers(p)
    um = [u[0] / p.b110 + b13 * u[2], u[1] / p.b220, u[2] / p.b330]
    div = k1 * um[0] + k2 * um[1] + k3 * um[2]
    assert np.abs(div).max() < 1e-12 * max(np.abs(c).max() for c in u)
    _, tke, eps = o.stats()
    assert tke > 0.0 and eps > 0.0


def test_rconv_equals_rrot_without_aliasing():
    """The convective product (u . D) u of R-conv and the rotational one w x u of R-rot
    differ by the laboratory gradient D(|u|^2 / 2), which the R-rot pressure term
    (shared by both forms, src/pf_rk3.f90:2089-2093) projects out.  For a field with
    moving-frame wavenumbers |k_d| <= N/6 the products are not aliased, so one stage of
    the two forms agrees to round-off, in a frame with bmat(1,3) != 0."""
    import oracle as O
    from pandora.params import workload_params
    p = workload_params("shear", 32)
    p.f_remesh_t, p.p_track_part, p.ns_deformed = 5, 0, 3
    o = O.Oracle(p)
    o.init_fluid()
    u = o.get_state()
    k1, k2, k3 = wavenumbers(p)
    keep = (np.abs(k1) <= 32 // 6) & (np.abs(k2) <= 32 // 6) & (np.abs(k3) <= 32 // 6)
    u = [np.where(keep, c, 0.0) for c in u]
    out = {}
    for form in (2, 3):
        q = p.copy()
        q.ns_deformed = form
        o2 = O.Oracle(q)
        o2.update_b(5, 0.3)
        assert o2.frame()[0] != 0.0
        o2.set_state(u)
        o2.stage(1, 5, 0.5 / p.f_deform_s / p.f_remesh_t)
        out[form] = o2.get_state()
    scale = max(np.abs(c).max() for c in out[3])
    diff = max(np.abs(a - b).max() for a, b in zip(out[2], out[3]))
    assert diff < 1e-13 * scale, diff / scale
    # while the two products themselves differ by that gradient
    nl = {}
    for form in (2, 3):
        q = p.copy()
        q.ns_deformed = form
        o2 = O.Oracle(q)
        o2.update_b(5, 0.3)
        o2.set_state(u)
        nl[form] = o2.nonlinear()
    gap = max(np.abs(a - b).max() for a, b in zip(nl[2], nl[3]))
    assert gap > 1e-2 * max(np.abs(c).max() for c in nl[3])

