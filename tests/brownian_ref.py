"""NumPy restatement of the rigid-body Brownian step (test infrastructure only).

Mirrors the library's cr_body_force_torque / cr_brownian_step: bead forces summed into
body forces and torques about the centres (minimum image), overdamped translation and
rotation with Stokes mobilities 1/(6 pi eta a) and 1/(8 pi eta a^3), Rodrigues
rotation about the centre, positions wrapped into [-L/2, L/2).  The Gaussian numbers
are SplitMix64 counters of (seed, step, body, component) through Box-Muller.
"""
from __future__ import annotations

import numpy as np

M64 = (1 << 64) - 1


def mix64(z: int) -> int:
    z = (z + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def unit_uniform(seed: int, step: int, body: int, k: int) -> float:
    z = mix64(seed ^ mix64((step * 0x100000001B3 + 0x51) & M64))
    z = mix64(z ^ ((body & 0xFFFFFFFF) << 8) ^ k)
    return (float(z >> 11) + 1.0) * (1.0 / 9007199254740992.0)


def normals6(seed: int, step: int, body: int) -> np.ndarray:
    g = np.empty(6)
    for k in range(3):
        u1 = unit_uniform(seed, step, body, 2 * k)
        u2 = unit_uniform(seed, step, body, 2 * k + 1)
        r = np.sqrt(-2.0 * np.log(u1))
        g[2 * k] = r * np.cos(2.0 * np.pi * u2)
        g[2 * k + 1] = r * np.sin(2.0 * np.pi * u2)
    return g


def _mimg(d, L):
    return d - L * np.rint(d / L)


def _wrap(x, L):
    return x - L * np.floor((x + 0.5 * L) / L)


def body_force_torque(pos, body, body_pos, force, L):
    L = np.asarray(L, dtype=np.float64)
    r = _mimg(pos - body_pos[body], L)
    B = len(body_pos)
    bf = np.zeros((B, 3))
    bt = np.zeros((B, 3))
    np.add.at(bf, body, force)
    np.add.at(bt, body, np.cross(r, force))
    return bf, bt


def rotation(th):
    ang = np.linalg.norm(th)
    if ang == 0.0:
        return np.eye(3), 0.0
    k = th / ang
    K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return np.eye(3) + np.sin(ang) * K + (1.0 - np.cos(ang)) * (K @ K), ang


def repulsion(body_pos, radius, L, k, gap):
    """Harmonic steric repulsion force on every body (all pairs, minimum image)."""
    D = _mimg(body_pos[None, :, :] - body_pos[:, None, :], L)   # D[b, j] = R_j - R_b
    d = np.linalg.norm(D, axis=-1)
    reach = radius[:, None] + radius[None, :] + gap
    on = (d < reach) & (d > 0)
    mag = np.where(on, k * (reach - d) / np.where(on, d, 1.0), 0.0)
    return -(mag[..., None] * D).sum(1)


def brownian_step(pos, body, rigid, body_pos, radius, force, L, step, dt=1e-3, kT=1.0, viscosity=1.0, seed=1,
                  k_rep=0.0, gap=0.0):
    """Returns new (pos, body_pos, moves[B, 2] = (|dR|, |dtheta|))."""
    L = np.asarray(L, dtype=np.float64)
    bf, bt = body_force_torque(pos, body, body_pos, force, L)
    if k_rep > 0:
        bf = bf + repulsion(body_pos, np.asarray(radius, dtype=np.float64), L, k_rep, gap)
    new_pos = np.empty_like(pos)
    new_bpos = np.empty_like(body_pos)
    moves = np.zeros((len(body_pos), 2))
    for b in range(len(body_pos)):
        a = radius[b]
        mt = 1.0 / (6.0 * np.pi * viscosity * a)
        mr = 1.0 / (8.0 * np.pi * viscosity * a ** 3)
        g = normals6(seed, step, b)
        dR = mt * bf[b] * dt + np.sqrt(2.0 * kT * mt * dt) * g[:3]
        th = mr * bt[b] * dt + np.sqrt(2.0 * kT * mr * dt) * g[3:] if rigid[b] else np.zeros(3)
        R, ang = rotation(th)
        c = body_pos[b] + dR
        idx = np.nonzero(body == b)[0]
        r = _mimg(pos[idx] - body_pos[b], L)
        new_pos[idx] = _wrap(c + r @ R.T, L)
        new_bpos[b] = _wrap(c, L)
        moves[b] = (np.linalg.norm(dR), ang)
    return new_pos, new_bpos, moves
