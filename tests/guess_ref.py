"""NumPy restatement of the learned-guess inputs (test infrastructure only).

Mirrors cr_guess_features: the surface gradient of the previous charges from the bead's
same-body neighbours ((D^T D + 1e-3 tr(D^T D) I) G = D^T dq), the transport term
s = G . (bead displacement - centre displacement), and the 48 features.  Neighbour sets
are taken as given; the tests check them separately against sorted distances.
"""
from __future__ import annotations

import numpy as np


def mimg(d, L):
    L = np.asarray(L, dtype=np.float64)
    return d - L * np.rint(d / L)


def features(q_prev, pos_prev, bpos_prev, pos, bpos, body, Q, radius, bead_nbr, body_nbr, E, L):
    N = len(pos)
    E = np.asarray(E, dtype=np.float64)
    D = mimg(pos_prev[bead_nbr] - pos_prev[:, None, :], L)              # [N, 6, 3]
    self_nbr = bead_nbr == np.arange(N)[:, None]
    D[self_nbr] = 0.0
    dq = q_prev[bead_nbr] - q_prev[:, None]
    dq[self_nbr] = 0.0
    A = np.einsum("nki,nkj->nij", D, D)
    rhs = np.einsum("nki,nk->ni", D, dq)
    eps = 1e-3 * np.trace(A, axis1=1, axis2=2) + 1e-300
    A = A + eps[:, None, None] * np.eye(3)
    G = np.linalg.solve(A, rhs[..., None])[..., 0]
    n = mimg(pos - bpos[body], L)
    n /= np.linalg.norm(n, axis=1)[:, None]
    delta = mimg((pos - pos_prev) - (bpos[body] - bpos_prev[body]), L)
    s = (G * delta).sum(1)
    f = np.zeros((N, 48))
    f[:, 0] = q_prev
    f[:, 1] = s
    f[:, 2] = n @ E
    f[:, 3] = Q[body]
    for k in range(body_nbr.shape[1]):
        j = body_nbr[body, k]
        u = mimg(bpos[j] - bpos[body], L)
        up = mimg(bpos_prev[j] - bpos_prev[body], L)
        d = np.linalg.norm(u, axis=1)
        dp = np.linalg.norm(up, axis=1)
        ok = (j != body) & (d > 0)
        c = np.where(ok, (n * u).sum(1) / np.where(ok, d, 1.0), 0.0)
        gap = np.maximum(d - radius[body] - radius[j], 0.0)
        w = 1.0 / (1.0 + gap)
        dg = 100.0 * (d - dp)
        g = np.stack([c, w, dg, dg * w * c, q_prev * dg], 1)
        g[~ok] = 0.0
        f[:, 4 + 5 * k:9 + 5 * k] = g
        if k == 0:
            f[:, 44] = np.where(ok, (u @ E) / np.where(ok, d, 1.0) * w, 0.0)
    return f, s
