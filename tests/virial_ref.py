"""NumPy restatement of the virial of U = 1/2 q.(M q) (test reference for cr_virial).

Real space: 1/2 sum_{i != j} r_ij (x) F_ij over the oracle's neighbour list with the pair
force of the reference's real_space_force (ConductorRigid.cu:637-654: the gradient table,
index floor(Ntable (d - dr)/(rc - dr)) and weight d/dr - index - 1, pairs with
dr^2 <= d^2 < rc^2).  Wave space: the spread mesh of the oracle (cu:144-234), its full
transform H(k), the oracle's influence function S(k) (cc:245-274), E_k = 1/2 h^3 S |H|^2
and -dE_k/de_ab = E_k (delta_ab + g k_a k_b / k^2), g = 2 k cot k - 4 - k^2/(2 xi^2).
"""
from __future__ import annotations

import numpy as np

import oracle


def _tensor6(V):
    return np.array([V[0, 0], V[0, 1], V[0, 2], V[1, 1], V[1, 2], V[2, 2]])


def real_virial(p, pos, L, q) -> np.ndarray:
    pos = np.asarray(pos, dtype=np.float64)
    L = np.asarray(L, dtype=np.float64)
    count, head, lst = oracle.neighbor_list(pos, L, p.rc)
    _, grad = oracle.tables(p)
    i = np.repeat(np.arange(len(pos)), count)
    j = lst
    d = pos[i] - pos[j]
    d -= L * np.rint(d * (1.0 / L))
    d2 = (d * d).sum(1)
    keep = (d2 < p.rc * p.rc) & (d2 >= p.dr * p.dr)
    i, j, d, d2 = i[keep], j[keep], d[keep], d2[keep]
    r = np.sqrt(d2)
    scale = p.N_table / (p.rc - p.dr)
    ind = np.clip(np.floor((r - p.dr) * scale).astype(np.int64), 0, p.N_table - 1)
    lin = r / p.dr - ind - 1.0
    Tp = grad[ind, 0] + (grad[ind, 1] - grad[ind, 0]) * lin
    a = -Tp * q[i] * q[j] / r
    V = 0.5 * np.einsum("n,na,nb->ab", a, d, d)
    return V


def real_pairs(p, pos, L):
    """Directed in-range pairs (i, j) with dr^2 <= d^2 < rc^2 under the minimum image."""
    pos = np.asarray(pos, dtype=np.float64)
    L = np.asarray(L, dtype=np.float64)
    count, head, lst = oracle.neighbor_list(pos, L, p.rc)
    i = np.repeat(np.arange(len(pos)), count)
    j = lst
    d = pos[i] - pos[j]
    d -= L * np.rint(d * (1.0 / L))
    d2 = (d * d).sum(1)
    keep = (d2 < p.rc * p.rc) & (d2 >= p.dr * p.dr)
    return i[keep], j[keep]


def real_energy_fixed_pairs(p, pos, L, q, i, j):
    """1/2 sum over the given directed pairs of q_i q_j T(d_ij) with the potential table
    (ConductorRigid.cu:549-554); the pair set is held fixed, so the energy is a continuous
    function of the positions (the truncated kernel itself jumps by T(rc-) at the cutoff)."""
    pos = np.asarray(pos, dtype=np.float64)
    L = np.asarray(L, dtype=np.float64)
    phi, _ = oracle.tables(p)
    d = pos[i] - pos[j]
    d -= L * np.rint(d * (1.0 / L))
    r = np.sqrt((d * d).sum(1))
    scale = p.N_table / (p.rc - p.dr)
    ind = np.clip(np.floor((r - p.dr) * scale).astype(np.int64), 0, p.N_table - 1)
    lin = r / p.dr - ind - 1.0
    T = phi[ind, 0] + (phi[ind, 1] - phi[ind, 0]) * lin
    return 0.5 * float((q[i] * q[j] * T).sum())


def wave_virial(p, pos, L, q):
    """(3x3 tensor, wave energy)."""
    g = oracle.spread(p, pos, q)
    H = np.fft.fftn(g)
    S = oracle.scale(p)
    E = 0.5 * p.quadW * S * np.abs(H) ** 2
    ks = [2.0 * np.pi * np.fft.fftfreq(p.N[d], d=1.0 / p.N[d]) / L[d] for d in range(3)]
    kx, ky, kz = np.meshgrid(*ks, indexing="ij")
    k2 = kx * kx + ky * ky + kz * kz
    k2[0, 0, 0] = 1.0
    k = np.sqrt(k2)
    s, c = np.sin(k), np.cos(k)
    cot = np.where(np.abs(s) > 1e-300, 2.0 * k * c / np.where(s == 0, 1.0, s), 0.0)
    gk = (cot - 4.0 - k2 / (2.0 * p.xi * p.xi)) / k2
    comps = [kx, ky, kz]
    V = np.zeros((3, 3))
    for a in range(3):
        for b in range(3):
            V[a, b] = float((E * ((1.0 if a == b else 0.0) + gk * comps[a] * comps[b])).sum())
    return V, float(E.sum())


def strained_energy(system, xi, errortol, grid, support, rcut, q, axis, delta):
    """U = 1/2 q.(M q) with positions and box stretched by (1 + delta) along `axis`."""
    import dataclasses

    f = np.ones(3)
    f[axis] += delta
    L = np.asarray(system.L, dtype=np.float64) * f
    pos = np.asarray(system.pos) * f
    pos = pos - L * np.floor((pos + 0.5 * L) / L)
    s2 = dataclasses.replace(system, L=L, pos=pos, body_pos=np.asarray(system.body_pos) * f)
    orc = oracle.Oracle(s2, xi, errortol, grid, support, rcut)
    return 0.5 * float(q @ orc.apply_M(q)), orc


def wave_energy_strained(system, xi, errortol, grid, support, rcut, q, axis, delta):
    _, orc = strained_energy(system, xi, errortol, grid, support, rcut, q, axis, delta)
    pos = orc.pos
    return 0.5 * float(q @ oracle.wave_potential(orc.p, pos, q))
