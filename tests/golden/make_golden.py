"""Generate tests/golden/*.npz with an independent NumPy/SciPy FP64 restatement.

This script restates the reference's algorithm a second time, in vectorised NumPy
(numpy.fft for the transform, scipy.special.erfc for the tables, brute-force pair
sums), independently of the C++ oracle, and records inputs and outputs for a small
system.  The tests compare the C++ oracle (and through it the CUDA product) with
these fixtures.  References are to the reference's files:

  SetParams            cppmodule/ConductorRigid.cc:116-207 (grid, P, eta)
  tables               cppmodule/ConductorRigid.cc:278-354
  influence function   cppmodule/ConductorRigid.cc:245-274
  spread / contract    cppmodule/ConductorRigid.cu:144-466
  real space           cppmodule/ConductorRigid.cu:469-664
  objective / precond  cppmodule/ConductorRigid.cu:764-859
  matvec               cppmodule/ConductorRigid.cu:862-1020

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np
from scipy.special import erfc

OUT = Path(__file__).resolve().parent


def smooth_sizes():
    s = sorted({2 ** a * 3 ** b * 5 ** c for a in range(13) for b in range(8) for c in range(6)})
    return [m for m in s if 8 <= m <= 4096]


def derive(L, xi, tol, grid=None, P=None, rc=None):
    L = np.asarray(L, dtype=float)
    root = math.sqrt(-math.log(tol))
    rcut = rc if rc else root / xi
    kcut = 2.0 * xi * root
    N = []
    for d in range(3):
        if grid:
            N.append(int(grid))
            continue
        n = int(math.ceil(1.0 + L[d] * kcut / math.pi))
        n = next(m for m in smooth_sizes() if n <= m)
        N.append(n)
    h = L / np.array(N, dtype=float)
    Pu = int(P) if P else int(math.ceil(-2.0 * math.log(tol) / math.pi))
    eta = Pu * h * h * xi * xi / math.pi
    Pc = min(Pu, *N)
    dr = 0.001
    nt = int(rcut / dr - 1)
    xiterm = 2.0 * xi * xi
    prefac = xiterm * xi / math.pi * math.sqrt(2.0 / (math.pi * eta[0] * eta[1] * eta[2]))
    quadW = float(h[0] * h[1] * h[2])
    selfc = (1.0 - math.exp(-4.0 * xi * xi)) / (8.0 * math.pi * math.sqrt(math.pi) * xi) + \
        math.erfc(2.0 * xi) / (4.0 * math.pi)
    return dict(L=L, xi=xi, N=np.array(N), P=Pc, P_unclamped=Pu, h=h, eta=eta, rc=rcut, kcut=kcut, N_table=nt,
                dr=dr, xiterm=xiterm, prefac=prefac, quadW=quadW, selfcoeff=selfc)


def tables(p):
    xi = p["xi"]
    xi2 = xi * xi
    r = (np.arange(p["N_table"] + 1) + 1) * p["dr"]
    r2 = r * r
    ep, em, e0 = np.exp(-(r + 2) ** 2 * xi2), np.exp(-(r - 2) ** 2 * xi2), np.exp(-r2 * xi2)
    cp, cm, c0 = erfc((r + 2) * xi), erfc((r - 2) * xi), erfc(r * xi)
    pi15 = math.pi ** 1.5
    pot = (-(r + 2) / (32 * pi15 * xi * r) * ep - (r - 2) / (32 * pi15 * xi * r) * em + 1 / (16 * pi15 * xi) * e0
           + (2 * xi2 * (r + 2) ** 2 + 1) / (64 * math.pi * xi2 * r) * cp
           + (2 * xi2 * (r - 2) ** 2 + 1) / (64 * math.pi * xi2 * r) * cm
           - (2 * xi2 * r2 + 1) / (32 * math.pi * xi2 * r) * c0
           + np.where(r < 2, -1 / (4 * math.pi * r) + (4 - r) / (16 * math.pi), 0.0))
    grad = (-(r - 2) / (32 * pi15 * xi * r2) * ep - (r + 2) / (32 * pi15 * xi * r2) * em
            + 1 / (16 * pi15 * xi * r) * e0
            + (2 * xi2 * r2 - 8 * xi2 - 1) / (64 * math.pi * xi2 * r2) * (cp + cm)
            - (2 * xi2 * r2 - 1) / (32 * math.pi * xi2 * r2) * c0
            + np.where(r < 2, 1 / (4 * math.pi * r2) - 1 / (16 * math.pi), 0.0))
    T1 = np.stack([pot, np.r_[pot[1:], 0.0]], axis=1)
    T2 = np.stack([grad, np.r_[grad[1:], 0.0]], axis=1)
    return T1, T2


def scale(p):
    N, L, eta, xi = p["N"], p["L"], p["eta"], p["xi"]
    ks = []
    for d in range(3):
        i = np.arange(N[d])
        ks.append(np.where(i < (N[d] + 1) // 2, i, i - N[d]) * 2.0 * math.pi / L[d])
    kx, ky, kz = np.meshgrid(*ks, indexing="ij")
    k2 = kx * kx + ky * ky + kz * kz
    etak2 = (1 - eta[0]) * kx * kx + (1 - eta[1]) * ky * ky + (1 - eta[2]) * kz * kz
    with np.errstate(divide="ignore", invalid="ignore"):
        kk = np.sqrt(k2)
        S = (np.sin(kk) / kk) ** 2 * np.exp(-etak2 / (4 * xi * xi)) / k2 / float(np.prod(N))
    S[0, 0, 0] = 0.0
    return S


def windows(p, pos):
    """Per bead: node indices (P,) per dim (wrapped) and r = node - pos (P,) per dim."""
    P, N, L, h = p["P"], p["N"], p["L"], p["h"]
    idx, r = [], []
    for d in range(3):
        u = (pos[:, d] + 0.5 * L[d]) / L[d] * N[d]
        x = np.trunc(u).astype(int)
        start = x - P // 2 + 1 - (P % 2) * ((u - x) < 0.5)
        nodes = start[:, None] + np.arange(P)[None, :]
        r.append(h[d] * nodes - 0.5 * L[d] - pos[:, d][:, None])
        idx.append(np.where(nodes < 0, nodes + N[d], np.where(nodes > N[d] - 1, nodes - N[d], nodes)))
    return idx, r


def gauss(p, r):
    e = p["eta"]
    arg = (r[0][:, :, None, None] ** 2 / e[0] + r[1][:, None, :, None] ** 2 / e[1] + r[2][:, None, None, :] ** 2 / e[2])
    return np.exp(-p["xiterm"] * arg)


def spread(p, pos, q):
    idx, r = windows(p, pos)
    g = p["prefac"] * gauss(p, r) * q[:, None, None, None]
    grid = np.zeros(tuple(p["N"]))
    ii = (idx[0][:, :, None, None], idx[1][:, None, :, None], idx[2][:, None, None, :])
    np.add.at(grid, np.broadcast_arrays(*ii), g)
    return grid


def wave_grid(p, pos, q):
    grid = spread(p, pos, q)
    G = float(np.prod(p["N"]))
    return np.real(np.fft.ifftn(np.fft.fftn(grid) * scale(p)) * G)


def contract(p, pos, grid):
    idx, r = windows(p, pos)
    vals = grid[idx[0][:, :, None, None], idx[1][:, None, :, None], idx[2][:, None, None, :]]
    return p["quadW"] * p["prefac"] * np.sum(gauss(p, r) * vals, axis=(1, 2, 3))


def contract_force(p, pos, q, grid):
    idx, r = windows(p, pos)
    vals = grid[idx[0][:, :, None, None], idx[1][:, None, :, None], idx[2][:, None, None, :]]
    g = gauss(p, r) * vals
    e = p["eta"]
    F = np.zeros((len(q), 3))
    F[:, 0] = np.sum(g * (-r[0][:, :, None, None] / e[0]), axis=(1, 2, 3))
    F[:, 1] = np.sum(g * (-r[1][:, None, :, None] / e[1]), axis=(1, 2, 3))
    F[:, 2] = np.sum(g * (-r[2][:, None, None, :] / e[2]), axis=(1, 2, 3))
    return 2.0 * p["quadW"] * p["prefac"] * p["xiterm"] * q[:, None] * F


def pair_geometry(p, pos):
    L = p["L"]
    d = pos[:, None, :] - pos[None, :, :]
    d = d - L * np.rint(d * (1.0 / L))
    d2 = np.sum(d * d, axis=-1)
    mask = (d2 < p["rc"] ** 2) & (d2 >= p["dr"] ** 2)
    np.fill_diagonal(mask, False)
    return d, d2, mask


def lerp(p, T, dist):
    ind = np.floor(p["N_table"] * (dist - p["dr"]) / (p["rc"] - p["dr"])).astype(int)
    lin = dist / p["dr"] - ind - 1.0
    return T[ind, 0] + (T[ind, 1] - T[ind, 0]) * lin


def apply_M(p, pos, q):
    T1, _ = tables(p)
    phi = contract(p, pos, wave_grid(p, pos, q)) + p["selfcoeff"] * q
    _, d2, mask = pair_geometry(p, pos)
    i, j = np.nonzero(mask)
    vals = lerp(p, T1, np.sqrt(d2[i, j])) * q[j]
    np.add.at(phi, i, vals)
    return phi


def forces(p, pos, q, E0):
    _, T2 = tables(p)
    F = contract_force(p, pos, q, wave_grid(p, pos, q)) + q[:, None] * E0[None, :]
    d, d2, mask = pair_geometry(p, pos)
    i, j = np.nonzero(mask)
    dist = np.sqrt(d2[i, j])
    A = lerp(p, T2, dist)
    np.add.at(F, i, (-A * q[i] * q[j] / dist)[:, None] * d[i, j])
    return F


def matvec(p, pos, body, B, x):
    N = len(body)
    Mq = apply_M(p, pos, x[:N])
    y = np.zeros(N + B)
    y[:N] = x[N + body] - Mq
    np.add.at(y, N + body, x[:N])
    return y


def objective(p, pos, body, rigid, bpos, Q, E0):
    N = len(body)
    r = pos - bpos[body]
    r = r - p["L"] * np.rint(r / p["L"])
    rhs = np.r_[-(r @ E0), Q]
    rhs[:N][rigid[body] == 0] = 0.0
    return rhs


def precondition(body, rigid, B, x):
    N = len(body)
    size = np.bincount(body, minlength=B)
    return np.r_[-4 * math.pi * x[:N], np.where(rigid == 1, x[N:] / size, x[N:] / (4 * math.pi))]


def small_system():
    rng = np.random.default_rng(20261203)
    L = np.array([9.0, 9.5, 10.0])
    centres = np.array([[-2.0, -1.5, 0.5], [1.2, 2.0, -1.0], [2.5, -2.2, 3.1]])
    pos, body = [], []
    for b, c in enumerate(centres):
        v = rng.standard_normal((20, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        pos.append(c + v)
        body.append(np.full(20, b))
    # two free beads
    pos.append(np.array([[3.9, 4.4, -4.6], [-4.2, 0.3, -3.3]]))
    body.append(np.array([3, 4]))
    pos = np.concatenate(pos)
    pos = pos - L * np.floor((pos + 0.5 * L) / L)
    body = np.concatenate(body).astype(np.uint32)
    rigid = np.array([1, 1, 1, 0, 0], dtype=np.uint8)
    Q = np.array([0.0, 1.0, -0.5, 0.25, -0.75])
    bpos = np.r_[centres, pos[-2:]]
    E0 = np.array([0.3, -0.2, 1.0])
    return L, pos, body, rigid, Q, bpos, E0


def main():
    L, pos, body, rigid, Q, bpos, E0 = small_system()
    xi = math.sqrt(-math.log(1e-5)) / 4.0
    p = derive(L, xi, 1e-5, grid=24, P=9, rc=4.0)
    N, B = len(body), len(Q)
    rng = np.random.default_rng(7)
    x = rng.standard_normal(N + B)
    T1, T2 = tables(p)
    out = dict(
        L=L, pos=pos, body=body, rigid=rigid, Q=Q, body_pos=bpos, E0=E0, xi=xi, errortol=1e-5, grid=24, support=9,
        rcut=4.0, x=x,
        grid_spread=spread(p, pos, x[:N]),
        phi_wave=contract(p, pos, wave_grid(p, pos, x[:N])),
        Mq=apply_M(p, pos, x[:N]),
        y=matvec(p, pos, body, B, x),
        rhs=objective(p, pos, body, rigid, bpos, Q, E0),
        Px=precondition(body, rigid, B, x),
        force=forces(p, pos, x[:N], E0),
        table_phiq=T1[:-1], table_grad=T2[:-1],
        eta=p["eta"], prefac=p["prefac"], selfcoeff=p["selfcoeff"], N_table=p["N_table"],
    )
    np.savez_compressed(OUT / "small_system.npz", **out)
    # parameter derivation cases without overrides (cc:116-207)
    cases = [((16.12, 16.12, 16.12), 0.5, 1e-3), ((30.0, 20.0, 12.0), 0.7, 1e-5), ((50.0, 50.0, 50.0), 0.848, 1e-6),
             ((11.0, 13.0, 17.0), 1.0, 1e-4)]
    rows = []
    for Lc, xic, tolc in cases:
        q = derive(Lc, xic, tolc)
        rows.append(np.r_[Lc, xic, tolc, q["N"], q["P"], q["P_unclamped"], q["eta"], q["rc"], q["N_table"],
                          q["prefac"], q["selfcoeff"]])
    np.save(OUT / "derive_cases.npy", np.array(rows))
    print("wrote", OUT / "small_system.npz", OUT / "derive_cases.npy")


if __name__ == "__main__":
    main()
