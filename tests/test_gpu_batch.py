"""Batches (pandora_batch_*): every member's result equals the same simulation run
alone, bit for bit -- whatever else shares its launches, and whenever it was
admitted (continuous batching: members at different step numbers advance in the
same launches)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _alone(pandora, p, nsteps):
    with pandora.Simulation(p) as s:
        s.init_fluid()
        if p.p_track_part and p.p_np_global > 0:
            s.init_particles()
        for k in range(1, nsteps + 1):
            s.step(k)
        u = s.get_state()
        xp = s.get_particles()[0] if p.p_track_part and p.p_np_global > 0 else None
    return u, xp


def _member(base, seed, nu=None):
    q = base.copy()
    q.seed_fluid, q.seed_force, q.seed_particles = seed, 1000 + seed, 2000 + seed
    if nu is not None:
        q.f_nu = nu
    return q


def _same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


def test_batch_members_equal_alone_runs(gpu_lib):
    base = gpu_lib.workload_params("iso_decay", 32)
    members = [_member(base, 11, 0.01), _member(base, 12, 0.02), _member(base, 13, 0.005)]
    late = _member(base, 14, 0.015)
    with gpu_lib.Batch(base, 5) as b:
        slots = [b.admit(q) for q in members]
        b.step(4)
        sl = b.admit(late)                # joins while the others are at step 5
        b.step(6)
        b.sync()
        assert b.member_time(slots[0])[0] == 11 and b.member_time(sl)[0] == 7
        for q, s in zip(members, slots):
            assert _same(b.get_state(s), _alone(gpu_lib, q, 10)[0])
        assert _same(b.get_state(sl), _alone(gpu_lib, late, 6)[0])


def test_batch_two_launch_chunks_particles(gpu_lib):
    """34 slots (two launches of up to 32 members), forced flow with 256 tracers."""
    base = gpu_lib.workload_params("iso_forced_particles", 32)
    base.p_np_global = 256
    with gpu_lib.Batch(base, 34) as b:
        slots = [b.admit(_member(base, 100 + k)) for k in range(34)]
        b.step(3)
        b.sync()
        for k in (0, 31, 32, 33):
            u, xp = _alone(gpu_lib, _member(base, 100 + k), 3)
            assert _same(b.get_state(slots[k]), u), k
            assert np.array_equal(b.get_particles(slots[k])[0], xp), k


def test_batch_mixed_precision_and_slot_reuse(gpu_lib):
    base = gpu_lib.workload_params("iso_decay", 48)
    base.precision = gpu_lib.PREC_FP32_MIXED
    with gpu_lib.Batch(base, 2) as b:
        s0 = b.admit(_member(base, 21))
        s1 = b.admit(_member(base, 22))
        b.step(3)
        b.release(s0)
        s2 = b.admit(_member(base, 23))      # reuses the slot: a fresh simulation
        b.step(2)
        b.sync()
        assert _same(b.get_state(s1), _alone(gpu_lib, _member(base, 22), 5)[0])
        assert _same(b.get_state(s2), _alone(gpu_lib, _member(base, 23), 2)[0])


@pytest.mark.parametrize("form", [1, 3])
def test_batch_shear_across_remesh(gpu_lib, form):
    """BF-rot (1) and R-rot (3) members: the batched K1, x pass and K5b of each form."""
    base = gpu_lib.workload_params("shear", 32)
    base.p_track_part = 0
    base.f_remesh_t = 2                      # remesh at step 5
    base.ns_deformed = form
    with gpu_lib.Batch(base, 2) as b:
        s0 = b.admit(_member(base, 31))
        b.step(2)
        s1 = b.admit(_member(base, 32))
        b.step(5)
        b.sync()
        assert _same(b.get_state(s0), _alone(gpu_lib, _member(base, 31), 7)[0])
        assert _same(b.get_state(s1), _alone(gpu_lib, _member(base, 32), 5)[0])
        ek, tke, eps = b.last_step_stats(s0)
        assert tke > 0 and eps > 0 and np.all(np.isfinite(ek))


def test_batch_rejects_other_class_and_full(gpu_lib):
    base = gpu_lib.workload_params("iso_decay", 32)
    with gpu_lib.Batch(base, 1) as b:
        other = gpu_lib.workload_params("iso_decay", 48)
        with pytest.raises(gpu_lib.PandoraError):
            b.admit(other)
        b.admit(_member(base, 1))
        with pytest.raises(gpu_lib.PandoraError):
            b.admit(_member(base, 2))


def test_ensemble_server_results_same_alone(gpu_lib):
    """A small trace through the ensemble server (continuous batching, both precisions,
    isotropic and sheared, with and without tracers): every run's final state equals
    the same request run alone."""
    from pandora import ensemble
    trace = ensemble.make_trace(6, seed=3, rate=None, steps=10, particles=64, sizes=(32, 48))
    for k, r in enumerate(trace):
        r.arrival = 0.0 if k < 6 else 0.001 * k     # the later half joins running batches
    caps = {f"{n}/{p}": {"best": 2} for n in (32, 48) for p in (0, 1)}
    srv = ensemble.Server(8 << 30, caps, chunk=3, keep_state=True)
    res = srv.run(trace, realtime=False)
    srv.close()
    assert res["requests"] == len(trace) and res["p99_ms"] > 0
    for r in trace:
        u, _ = _alone(gpu_lib, r.params, r.steps)
        assert _same(r.result["u"], u), r.rid


def test_batch_rejects_other_forcing_radius(gpu_lib):
    """The forcing mask is kmag <= FORCE_KF, a real number: a member whose radius differs
    only in its fractional part is another class, not a member that would run with the
    batch's radius."""
    base = gpu_lib.workload_params("iso_forced_particles", 32)
    base.p_track_part = 0
    other = _member(base, 5)
    other.force_kf = 2.9                  # same aint(FORCE_KF) = 2 as the batch's 2.5
    with gpu_lib.Batch(base, 2) as b:
        with pytest.raises(gpu_lib.PandoraError):
            b.admit(other)
        assert gpu_lib.class_key(other) != gpu_lib.class_key(base)


def test_batch_many_outstanding_tickets(gpu_lib):
    """More tickets outstanding than the batch keeps events for: an old ticket is done
    only once its work is, and a finished member's statistics are readable then."""
    base = gpu_lib.workload_params("iso_decay", 32)
    with gpu_lib.Batch(base, 2) as b:
        s0 = b.admit(_member(base, 41))
        first = b.step(1)
        tickets = [b.step(1) for _ in range(600)]     # more than the 512 event slots
        fin = b.finish(s0)
        assert fin > tickets[-1] > first
        b.sync()
        assert b.done(first) and b.done(tickets[0]) and b.done(fin)
        ek, tke, eps = b.result_stats(s0)
        # the statistics of stage 1 of the member's last step (its 601st)
        u, _ = _alone(gpu_lib, _member(base, 41), 600)
        with gpu_lib.Simulation(_member(base, 41)) as s:
            s.set_state(u)
            ek2, tke2, eps2, _ = s.stats()
        assert tke == pytest.approx(tke2, rel=1e-12) and eps == pytest.approx(eps2, rel=1e-12)


def test_batch_integrating_factor_class(gpu_lib):
    """Members in the integrating-factor form run in a batch of their own class (one
    update kernel per launch) and equal their runs alone; an explicit member is refused."""
    base = gpu_lib.workload_params("iso_decay", 32)
    base.rk3_viscous = gpu_lib.VISCOUS_INTEGRATING_FACTOR
    a, b = _member(base, 51), _member(base, 52, 0.02)
    with gpu_lib.Batch(base, 2) as bt:
        sa = bt.admit(a)
        bt.step(2)
        sb = bt.admit(b)
        bt.step(3)
        bt.sync()
        assert _same(bt.get_state(sa), _alone(gpu_lib, a, 5)[0])
        assert _same(bt.get_state(sb), _alone(gpu_lib, b, 3)[0])
    ex = _member(base, 53)
    ex.rk3_viscous = gpu_lib.VISCOUS_EXPLICIT
    with gpu_lib.Batch(base, 1) as bt:
        with pytest.raises(gpu_lib.PandoraError):
            bt.admit(ex)


def test_batch_lengths_without_batched_kernels_refused(gpu_lib):
    """Lengths outside the ensemble's sizes have single-simulation kernels only: a batch
    of several members is refused, a batch of one runs them."""
    base = gpu_lib.workload_params("iso_decay", 80)
    with pytest.raises(gpu_lib.PandoraError) as ei:
        gpu_lib.Batch(base, 2)
    assert ei.value.status == -10
    with gpu_lib.Batch(base, 1) as b:
        s0 = b.admit(_member(base, 71))
        b.step(2)
        b.sync()
        assert _same(b.get_state(s0), _alone(gpu_lib, _member(base, 71), 2)[0])


@pytest.mark.parametrize("lpw", [2, 4])
def test_batch_x_lines_per_warp(gpu_lib, lpw):
    """A batch whose x pass runs several lines per warp: members equal their runs alone
    (with the default schedule) bit for bit."""
    base = gpu_lib.workload_params("iso_forced_particles", 32)
    base.p_np_global = 128
    cls = base.copy()
    cls.x_lines_per_warp = lpw
    with gpu_lib.Batch(cls, 3) as b:
        slots = [b.admit(_member(cls, 81 + k)) for k in range(3)]
        b.step(3)
        b.sync()
        for k, sl in enumerate(slots):
            u, xp = _alone(gpu_lib, _member(base, 81 + k), 3)
            assert _same(b.get_state(sl), u), k
            assert np.array_equal(b.get_particles(sl)[0], xp), k
