"""Shared helpers of the parity tests (relative errors, wavenumber grids)."""
import numpy as np


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    num = np.sqrt(sum(np.sum(np.abs(x - y) ** 2) for x, y in zip(np.atleast_1d(a), np.atleast_1d(b))))
    den = np.sqrt(sum(np.sum(np.abs(y) ** 2) for y in np.atleast_1d(b)))
    return float(num / den) if den > 0 else float(num)


def rel_l2_fields(us, vs) -> float:
    num = sum(float(np.sum(np.abs(u - v) ** 2)) for u, v in zip(us, vs))
    den = sum(float(np.sum(np.abs(v) ** 2)) for v in vs)
    return (num / den) ** 0.5 if den > 0 else num ** 0.5


def wavenumbers(p):
    ki, kj, kk = p.nodes_x // 3, p.nodes_y // 3, p.nodes_z // 3
    a = np.arange(ki + 1, dtype=float)
    b = np.arange(2 * kj + 1)
    b = np.where(b <= kj, b, b - (2 * kj + 1)).astype(float)
    c = np.arange(2 * kk + 1)
    c = np.where(c <= kk, c, c - (2 * kk + 1)).astype(float)
    return a[:, None, None], b[None, :, None], c[None, None, :]


def divergence(p, u):
    k1, k2, k3 = wavenumbers(p)
    return k1 * u[0] + k2 * u[1] + k3 * u[2]
