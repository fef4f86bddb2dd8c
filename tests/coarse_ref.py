"""Dense numpy restatement of the two-level conductor preconditioner (test-side checker).

Independent of the CUDA code: per rigid body the isolated-conductor block of the
saddle-point system with the free-space unit-shell kernel, the three induced-dipole
columns z_ba = A_b^-1 [-(r - r_b0).e_a; 0], the coarse operator
C = Z_q^T (self I + T + W_k) Z_q with T the tabulated real-space kernel under the
operator's pair rule (dr <= d < rc, minimum image; ConductorRigid.cu:536-557) and W_k
the wave-space kernel restricted to 0 < |k| < 2 xi (form factor j0(k)^2, Ewald factor
exp(-k^2/4xi^2), 1/(k^2 V); ConductorRigid.cc:245-274), and the A-DEF1 application
z = P (r - A~ Z y) + Z y with y = -C^-1 Z^T r.  With pcg_steps > 0 the sparse form:
y from that many block-Jacobi CG steps on C y = -Z^T r (the diagonal blocks include
the wave-space term).  Small systems only (dense N x N).
"""
import numpy as np


def _shell(D):
    K = np.where(D < 2, (4 - D) / (16 * np.pi), 1 / (4 * np.pi * np.maximum(D, 1e-300)))
    np.fill_diagonal(K, 1 / (4 * np.pi))
    return K


def _mimg(d, L):
    return d - L * np.rint(d / L)


class TwoLevelRef:
    def __init__(self, s, derived: dict, phiq: np.ndarray, xi: float, min_beads: int = 4, pcg_steps: int = 0):
        self.s = s
        N, B = s.n_beads, s.n_bodies
        L = np.asarray(s.L, dtype=float)
        self.N, self.B = N, B
        self.members = [np.nonzero(s.body == b)[0] for b in range(B)]
        # body blocks and their inverses
        self.Ainv = []
        for b in range(B):
            idx = self.members[b]
            d = _mimg(s.pos[idx][:, None, :] - s.pos[idx][None, :, :], L)
            K = _shell(np.linalg.norm(d, axis=-1))
            n = len(idx)
            A = np.zeros((n + 1, n + 1))
            A[:n, :n] = -K
            A[:n, n] = 1
            A[n, :n] = 1
            self.Ainv.append(np.linalg.inv(A))
        # coarse columns
        self.cbody = [b for b in range(B) if s.rigid[b] and len(self.members[b]) >= min_beads]
        nc = 3 * len(self.cbody)
        Z = np.zeros((N + B, nc))
        for a, b in enumerate(self.cbody):
            idx = self.members[b]
            rel = _mimg(s.pos[idx] - s.pos[idx[0]], L)
            for e in range(3):
                sol = self.Ainv[b] @ np.r_[-rel[:, e], 0.0]
                Z[idx, 3 * a + e] = sol[:-1]
                Z[N + b, 3 * a + e] = sol[-1]
        self.Z = Z
        Zq = Z[:N]
        # real-space kernel matrix
        rc, dr, ntab = derived["rcut"], derived["dr"], derived["n_table"]
        d = _mimg(s.pos[:, None, :] - s.pos[None, :, :], L)
        D = np.linalg.norm(d, axis=-1)
        ok = (D * D < rc * rc) & (D * D >= dr * dr)
        ind = np.clip(np.floor(ntab * (D - dr) / (rc - dr)).astype(np.int64), 0, ntab - 1)
        lin = D / dr - ind - 1.0
        T = np.where(ok, phiq[ind, 0] + (phiq[ind, 1] - phiq[ind, 0]) * lin, 0.0)
        # low-k wave kernel between beads
        V = float(np.prod(L))
        kc = 2.0 * xi
        mmax = np.floor(kc * L / (2 * np.pi)).astype(int)
        ks = []
        for mx in range(0, mmax[0] + 1):
            for my in range(-mmax[1], mmax[1] + 1):
                for mz in range(-mmax[2], mmax[2] + 1):
                    if mx == 0 and (my < 0 or (my == 0 and mz <= 0)):
                        continue
                    k = 2 * np.pi * np.array([mx, my, mz]) / L
                    kk = np.linalg.norm(k)
                    if kk < kc:
                        ks.append(k)
        self.pcg_steps = pcg_steps
        self.n_modes = len(ks)
        Wk = np.zeros((N, N))
        for k in ks:
            kk = np.linalg.norm(k)
            w = 2.0 * (np.sin(kk) / kk) ** 2 * np.exp(-kk * kk / (4 * xi * xi)) / (kk * kk * V)
            ph = s.pos @ k
            Wk += w * (np.cos(ph)[:, None] * np.cos(ph)[None, :] + np.sin(ph)[:, None] * np.sin(ph)[None, :])
        self.Mmodel = derived["selfcoeff"] * np.eye(N) + T + Wk
        self.C = Zq.T @ self.Mmodel @ Zq
        self.Cinv = np.linalg.inv(self.C)
        nb = nc // 3
        self.Dblk = [np.linalg.inv(0.5 * (self.C[3 * a:3 * a + 3, 3 * a:3 * a + 3] +
                                          self.C[3 * a:3 * a + 3, 3 * a:3 * a + 3].T)) for a in range(nb)]

    def _jacobi(self, r):
        z = np.empty_like(r)
        for a, D in enumerate(self.Dblk):
            z[3 * a:3 * a + 3] = D @ r[3 * a:3 * a + 3]
        return z

    def coarse_solve(self, g):
        """y = -C^-1 g: exact (dense form) or pcg_steps block-Jacobi CG steps (sparse form)."""
        if not self.pcg_steps:
            return -self.Cinv @ g
        y = np.zeros_like(g)
        r = -g
        z = self._jacobi(r)
        p = z.copy()
        rz = r @ z
        for it in range(self.pcg_steps):
            q = self.C @ p
            pq = p @ q
            alpha = rz / pq if pq > 0 else 0.0
            y += alpha * p
            r = r - alpha * q
            z = self._jacobi(r)
            rzn = r @ z
            if it + 1 < self.pcg_steps:
                beta = rzn / rz if rz > 0 else 0.0
                p = z + beta * p
            rz = rzn
        return y

    def conductor(self, v):
        N = self.N
        z = np.zeros_like(v)
        for b in range(self.B):
            idx = self.members[b]
            sol = self.Ainv[b] @ np.r_[v[idx], v[N + b]]
            z[idx] = sol[:-1]
            z[N + b] = sol[-1]
        return z

    def apply(self, r):
        N = self.N
        y = self.coarse_solve(self.Z.T @ r)
        zy = self.Z @ y
        t = r.copy()
        # A~ Z y = [Phi(Z y) - M~ (Z_q y); S Z_q y = 0]
        t[:N] -= zy[N + self.s.body] - self.Mmodel @ zy[:N]
        return self.conductor(t) + zy
