"""Restart files in the reference's PETSc binary format (no GPU): the byte layout,
round trips, the scaled copy of a coarser field."""
import numpy as np
import pytest

from pandora import restart


def test_vec_bytes_are_petsc_binary(tmp_path):
    """VecView to a binary viewer: class id 1211214, length, values, big-endian."""
    path = tmp_path / "vec.bin"
    with open(path, "wb") as fh:
        restart.write_vec(fh, np.array([1.0, -2.5]))
    raw = path.read_bytes()
    assert raw[:4] == (1211214).to_bytes(4, "big")
    assert raw[4:8] == (2).to_bytes(4, "big")
    assert raw[8:] == np.array([1.0, -2.5], dtype=">f8").tobytes()


def test_fluid_round_trip_and_layout(tmp_path):
    rng = np.random.default_rng(3)
    shape = (6, 11, 11)
    u = [rng.standard_normal(shape) + 1j * rng.standard_normal(shape) for _ in range(3)]
    f = tmp_path / "fluid.bin"
    restart.write_fluid(str(f), u)
    raw = np.fromfile(str(f), dtype=">f8", offset=8, count=4)
    # [i][j][k][re, im]: the first values are u1(0,0,0) re, im, then u1(0,0,1)
    assert np.array_equal(raw, [u[0][0, 0, 0].real, u[0][0, 0, 0].imag, u[0][0, 0, 1].real, u[0][0, 0, 1].imag])
    back = restart.read_fluid(str(f), shape)
    assert all(np.array_equal(a, b) for a, b in zip(u, back))
    with pytest.raises(ValueError):
        restart.read_fluid(str(f), (6, 11, 13))


def test_index64_header(tmp_path):
    f = tmp_path / "v.bin"
    with open(f, "wb") as fh:
        restart.write_vec(fh, np.arange(3.0), index64=True)
    with open(f, "rb") as fh:
        assert np.array_equal(restart.read_vec(fh, index64=True), np.arange(3.0))


def test_scaled_copy_keeps_wavenumbers():
    """A 16^3 field (K = 5) placed in the 32^3 layout (K = 10): every mode keeps its
    wavenumber, the rest is zero."""
    rng = np.random.default_rng(5)
    c_shape, f_shape = (6, 11, 11), (11, 21, 21)
    u = [rng.standard_normal(c_shape) + 1j * rng.standard_normal(c_shape) for _ in range(3)]
    f = restart.scale_fluid(u, f_shape)
    wv = lambda idx, K: idx if idx <= K else idx - (2 * K + 1)
    for i in range(6):
        for j in range(11):
            for k in range(11):
                jj, kk = wv(j, 5), wv(k, 5)
                fj = jj if jj >= 0 else jj + 21
                fk = kk if kk >= 0 else kk + 21
                assert f[1][i, fj, fk] == u[1][i, j, k]
    assert sum(np.count_nonzero(a) for a in f) == sum(np.count_nonzero(a) for a in u)


def test_particles_round_trip(tmp_path):
    rng = np.random.default_rng(7)
    xp, up = rng.random((3, 50)), rng.random((3, 50))
    dp = rng.random(50)
    f = tmp_path / "part.bin"
    restart.write_particles(str(f), xp, up, dp, xp0=xp)
    d = restart.read_particles(str(f), keep_initial=True)
    assert np.array_equal(d["xp2"], xp[1]) and np.array_equal(d["up3"], up[2]) and np.array_equal(d["dp"], dp)
    assert np.array_equal(d["status"], np.zeros(50)) and np.array_equal(d["xp03"], xp[2])


@pytest.mark.gpu
def test_simulation_restart_round_trip(gpu_lib, tmp_path):
    """Write a running simulation's restart files, read them into a fresh one (and a
    16^3 field into a 32^3 simulation with F_RESTART_SCALE = 2)."""
    p = gpu_lib.workload_params("iso_forced_particles", 32)
    p.p_np_global = 300
    with gpu_lib.Simulation(p) as a:
        a.init_fluid()
        a.init_particles()
        a.advance(3)
        a.write_restart(str(tmp_path / "f.bin"), str(tmp_path / "p.bin"))
        ua = a.get_state()
        xa, upa, _, _, dpa = a.get_particles()
    with gpu_lib.Simulation(p) as b:
        b.read_restart(str(tmp_path / "f.bin"), str(tmp_path / "p.bin"))
        assert all(np.array_equal(x, y) for x, y in zip(ua, b.get_state()))
        xb, upb, _, _, dpb = b.get_particles()
        assert np.array_equal(xa, xb) and np.array_equal(upa, upb) and np.array_equal(dpa, dpb)
    q = gpu_lib.workload_params("iso_decay", 16)
    with gpu_lib.Simulation(q) as c:
        c.init_fluid()
        c.write_restart(str(tmp_path / "c.bin"))
        uc = c.get_state()
    r = gpu_lib.workload_params("iso_decay", 32)
    with gpu_lib.Simulation(r) as d:
        d.read_restart(str(tmp_path / "c.bin"), scale=2)
        want = restart.scale_fluid(uc, d.shape)
        assert all(np.array_equal(x, y) for x, y in zip(want, d.get_state()))

