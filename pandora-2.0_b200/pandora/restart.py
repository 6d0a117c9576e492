"""Restart files in the reference's format: PETSc binary vectors.

g_RestartPetscFluid (src/pg_restart.f90:39-190) writes u1, u2, u3 with VecView to one
binary viewer (no info file): each vector is the class id 1211214 (VEC_FILE_CLASSID),
its global length, then its values, all big-endian (int32 header words; int64
length for a PETSc built with 64-bit indices), and a DMDA vector goes out in the
DMDA's natural order, which for the spectral velocity (dof 2 = re, im; k fastest,
then j, then i) is the reference layout [i][j][k][re, im] itself.
g_RestartPetscParticle (src/pg_restart.f90:192-330) writes xp1..3, up1..3, dp and
status (and xp01..03 with P_KEEP_INITIAL_POSITION) the same way, one value per
particle, in the order the ranks hold them.

A scaled restart (F_RESTART_SCALE > 1, f_InitialiseCopyRestart,
src/pf_initialise.f90:1184-1299) reads the field of a grid `scale` times coarser and
places every stored mode at the same wavenumber of the finer layout, zero
elsewhere.  (The reference's loop takes either the positive or the negative j
half, depending on where a rank's j range starts, so a single-rank reference run
copies only j >= 0; here both halves are copied.)
"""
from __future__ import annotations

import numpy as np

VEC_FILE_CLASSID = 1211214


def write_vec(fh, values: np.ndarray, index64: bool = False) -> None:
    v = np.ascontiguousarray(values, dtype=">f8").ravel()
    np.array([VEC_FILE_CLASSID], dtype=">i4").tofile(fh)
    np.array([v.size], dtype=">i8" if index64 else ">i4").tofile(fh)
    v.tofile(fh)


def read_vec(fh, index64: bool = False) -> np.ndarray:
    head = np.fromfile(fh, dtype=">i4", count=1)
    if head.size != 1 or int(head[0]) != VEC_FILE_CLASSID:
        raise ValueError("not a PETSc binary vector (class id mismatch)")
    n = np.fromfile(fh, dtype=">i8" if index64 else ">i4", count=1)
    if n.size != 1 or n[0] < 0:
        raise ValueError("truncated PETSc vector header")
    v = np.fromfile(fh, dtype=">f8", count=int(n[0]))
    if v.size != int(n[0]):
        raise ValueError("truncated PETSc vector")
    return v.astype(np.float64)


def _interleave(u: np.ndarray) -> np.ndarray:
    out = np.empty(u.shape + (2,), dtype=np.float64)
    out[..., 0] = u.real
    out[..., 1] = u.imag
    return out


def write_fluid(path: str, u, index64: bool = False) -> None:
    """u: three complex arrays [i][j][k] (the state of `Simulation.get_state()`)."""
    with open(path, "wb") as fh:
        for c in range(3):
            write_vec(fh, _interleave(np.asarray(u[c])), index64)


def read_fluid(path: str, shape, index64: bool = False):
    """Three complex arrays of `shape` = (NKI, NKJ, NKK) from a fluid restart file."""
    n = int(np.prod(shape))
    out = []
    with open(path, "rb") as fh:
        for _ in range(3):
            v = read_vec(fh, index64)
            if v.size != 2 * n:
                raise ValueError(f"restart vector has {v.size // 2} modes, the grid {n}")
            v = v.reshape(tuple(shape) + (2,))
            out.append(v[..., 0] + 1j * v[..., 1])
    return out


def scale_fluid(u_coarse, fine_shape):
    """f_InitialiseCopyRestart: the coarse spectrum at the same wavenumbers of the
    finer layout (both j and k halves), zero elsewhere."""
    nki_c, nkj_c, nkk_c = u_coarse[0].shape
    nki, nkj, nkk = fine_shape
    kj_c, kk_c = (nkj_c - 1) // 2, (nkk_c - 1) // 2
    jmap = np.array([j if j <= kj_c else nkj - (nkj_c - j) for j in range(nkj_c)])
    kmap = np.array([k if k <= kk_c else nkk - (nkk_c - k) for k in range(nkk_c)])
    out = []
    for c in range(3):
        f = np.zeros(fine_shape, dtype=np.complex128)
        f[np.ix_(np.arange(min(nki_c, nki)), jmap, kmap)] = u_coarse[c][: min(nki_c, nki)]
        out.append(f)
    return out


PARTICLE_FIELDS = ("xp1", "xp2", "xp3", "up1", "up2", "up3", "dp", "status")


def write_particles(path: str, xp: np.ndarray, up: np.ndarray, dp: np.ndarray, status=None, xp0=None,
                    index64: bool = False) -> None:
    """xp, up: [3][np]; dp: [np]; status: [np] (0 = active, the default); xp0: the
    initial positions [3][np] when the run keeps them."""
    npart = np.asarray(dp).size
    st = np.zeros(npart) if status is None else np.asarray(status, dtype=np.float64)
    with open(path, "wb") as fh:
        for a in (xp[0], xp[1], xp[2], up[0], up[1], up[2], dp, st):
            write_vec(fh, np.asarray(a, dtype=np.float64), index64)
        if xp0 is not None:
            for a in xp0:
                write_vec(fh, np.asarray(a, dtype=np.float64), index64)


def read_particles(path: str, keep_initial: bool = False, index64: bool = False) -> dict:
    out = {}
    with open(path, "rb") as fh:
        for name in PARTICLE_FIELDS:
            out[name] = read_vec(fh, index64)
        if keep_initial:
            for name in ("xp01", "xp02", "xp03"):
                out[name] = read_vec(fh, index64)
    n = out["dp"].size
    if any(v.size != n for v in out.values()):
        raise ValueError("particle restart vectors differ in length")
    return out
