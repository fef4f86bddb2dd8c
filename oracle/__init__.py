"""FP64 CPU oracle of ConductorRigid's induced-charge solve (TEST INFRASTRUCTURE).

Python side of oracle/cr_oracle.{h,cc}.  Only tests/, ``__graft_entry__.smoke()``
and bench.py's CPU-baseline leg may import this package; the product never does.

Parity unpinned against reference outputs: the reference (a HOOMD-blue 1.x plugin)
needs HOOMD, CUSP and Boost and uses CUDA texture references removed in CUDA 12, so
it cannot be built or run here, and it ships no tests or golden vectors.  The
restatement is pinned by the known-answer tests under tests/ instead.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libcr_oracle.so"

_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)
_IP = C.POINTER(C.c_int)


class OrcParams(C.Structure):
    _fields_ = [
        ("L", C.c_double * 3),
        ("xi", C.c_double),
        ("errortol", C.c_double),
        ("grid_override", C.c_int * 3),
        ("support_override", C.c_int),
        ("rc_override", C.c_double),
        ("N", C.c_int * 3),
        ("P", C.c_int),
        ("P_unclamped", C.c_int),
        ("h", C.c_double * 3),
        ("eta", C.c_double * 3),
        ("rc", C.c_double),
        ("kcut", C.c_double),
        ("N_table", C.c_int),
        ("dr", C.c_double),
        ("selfcoeff", C.c_double),
        ("xiterm", C.c_double),
        ("prefac", C.c_double),
        ("quadW", C.c_double),
    ]


_lib = None


def build() -> Path:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    r = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        sigs = {
            "orc_derive": ([C.POINTER(OrcParams)], C.c_int),
            "orc_tables": ([C.POINTER(OrcParams), _D, _D], None),
            "orc_scale": ([C.POINTER(OrcParams), _D], None),
            "orc_fft3d": ([C.c_int, C.c_int, C.c_int, _D, _D, C.c_int], None),
            "orc_spread": ([C.POINTER(OrcParams), C.c_int, _D, _D, _D], None),
            "orc_contract": ([C.POINTER(OrcParams), C.c_int, _D, _D, _D], None),
            "orc_contract_force": ([C.POINTER(OrcParams), C.c_int, _D, _D, _D, _D], None),
            "orc_wave_potential": ([C.POINTER(OrcParams), C.c_int, _D, _D, _D], None),
            "orc_wave_force": ([C.POINTER(OrcParams), C.c_int, _D, _D, _D], None),
            "orc_neighbor_list": ([C.c_int, _D, _D, C.c_double, _IP, _I64, _IP], C.c_int64),
            "orc_create": ([C.POINTER(OrcParams), C.c_int, C.c_int, C.POINTER(C.c_uint32),
                            C.POINTER(C.c_uint8), _D], C.c_void_p),
            "orc_destroy": ([C.c_void_p], None),
            "orc_set_positions": ([C.c_void_p, _D, _D], C.c_int),
            "orc_apply_M": ([C.c_void_p, _D, _D], None),
            "orc_matvec": ([C.c_void_p, _D, _D], None),
            "orc_precondition": ([C.c_void_p, _D, _D], None),
            "orc_objective": ([C.c_void_p, _D, _D], None),
            "orc_gmres": ([C.c_void_p, _D, _D, C.c_int, C.c_int, C.c_double, _D, _D], C.c_int),
            "orc_forces": ([C.c_void_p, _D, _D, _D], None),
            "orc_solve": ([C.c_void_p, _D, _D, _D, _D, C.c_int, C.c_int, C.c_double, _D], C.c_int),
            "orc_num_threads": ([], C.c_int),
        }
        for name, (a, r) in sigs.items():
            f = getattr(L, name)
            f.argtypes = a
            f.restype = r
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def c64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def derive(L, xi, errortol, grid=None, support=0, rcut=0.0) -> OrcParams:
    p = OrcParams()
    p.L[:] = [float(v) for v in np.broadcast_to(np.asarray(L, dtype=float), (3,))]
    p.xi = float(xi)
    p.errortol = float(errortol)
    g = [0, 0, 0] if grid is None else ([int(grid)] * 3 if np.isscalar(grid) else [int(v) for v in grid])
    p.grid_override[:] = g
    p.support_override = int(support)
    p.rc_override = float(rcut)
    st = lib().orc_derive(C.byref(p))
    if st != 0:
        raise ValueError(f"orc_derive failed with code {st}")
    return p


def params_dict(p: OrcParams) -> dict:
    return {name: (list(getattr(p, name)) if hasattr(getattr(p, name), "__len__") else getattr(p, name))
            for name, _ in p._fields_}


def tables(p: OrcParams):
    n = p.N_table + 1
    a, b = np.zeros(2 * n), np.zeros(2 * n)
    lib().orc_tables(C.byref(p), _dp(a), _dp(b))
    return a.reshape(n, 2), b.reshape(n, 2)


def scale(p: OrcParams) -> np.ndarray:
    s = np.zeros(p.N[0] * p.N[1] * p.N[2])
    lib().orc_scale(C.byref(p), _dp(s))
    return s.reshape(p.N[0], p.N[1], p.N[2])


def fft3d(re, im, sign: int):
    re, im = c64(re).copy(), c64(im).copy()
    n0, n1, n2 = re.shape
    lib().orc_fft3d(n0, n1, n2, _dp(re), _dp(im), int(sign))
    return re, im


def spread(p: OrcParams, pos, q) -> np.ndarray:
    pos, q = c64(pos), c64(q)
    g = np.zeros(p.N[0] * p.N[1] * p.N[2])
    lib().orc_spread(C.byref(p), len(q), _dp(pos), _dp(q), _dp(g))
    return g.reshape(p.N[0], p.N[1], p.N[2])


def contract(p: OrcParams, pos, grid) -> np.ndarray:
    pos, grid = c64(pos), c64(grid)
    out = np.zeros(pos.shape[0])
    lib().orc_contract(C.byref(p), pos.shape[0], _dp(pos), _dp(grid), _dp(out))
    return out


def wave_potential(p: OrcParams, pos, q) -> np.ndarray:
    pos, q = c64(pos), c64(q)
    out = np.zeros(len(q))
    lib().orc_wave_potential(C.byref(p), len(q), _dp(pos), _dp(q), _dp(out))
    return out


def wave_force(p: OrcParams, pos, q) -> np.ndarray:
    pos, q = c64(pos), c64(q)
    out = np.zeros(3 * len(q))
    lib().orc_wave_force(C.byref(p), len(q), _dp(pos), _dp(q), _dp(out))
    return out.reshape(-1, 3)


def neighbor_list(pos, L, r_list: float):
    """CSR (count, head, list) of every j != i within r_list, per-bead ascending."""
    pos = c64(pos)
    Lv = c64(np.broadcast_to(np.asarray(L, dtype=float), (3,)))
    N = pos.shape[0]
    count = np.zeros(N, dtype=np.int32)
    head = np.zeros(N, dtype=np.int64)
    tot = lib().orc_neighbor_list(N, _dp(pos), _dp(Lv), float(r_list), count.ctypes.data_as(_IP),
                                  head.ctypes.data_as(_I64), None)
    lst = np.zeros(max(tot, 1), dtype=np.int32)
    lib().orc_neighbor_list(N, _dp(pos), _dp(Lv), float(r_list), count.ctypes.data_as(_IP),
                            head.ctypes.data_as(_I64), lst.ctypes.data_as(_IP))
    return count, head, lst[:tot]


class Oracle:
    """Solver context over one system (positions fixed until set_positions)."""

    def __init__(self, system, xi, errortol, grid=None, support=0, rcut=0.0):
        self.p = derive(system.L, xi, errortol, grid, support, rcut)
        self.N = system.n_beads
        self.B = system.n_bodies
        body = np.ascontiguousarray(system.body, dtype=np.uint32)
        rigid = np.ascontiguousarray(system.rigid, dtype=np.uint8)
        Q = c64(system.body_charge)
        self.ctx = lib().orc_create(C.byref(self.p), self.N, self.B, body.ctypes.data_as(C.POINTER(C.c_uint32)),
                                    rigid.ctypes.data_as(C.POINTER(C.c_uint8)), _dp(Q))
        self.system = system
        self.set_positions(system.pos, system.body_pos)

    def __del__(self):
        try:
            if getattr(self, "ctx", None):
                lib().orc_destroy(self.ctx)
                self.ctx = None
        except Exception:
            pass

    def set_positions(self, pos, body_pos):
        self.pos = c64(pos)
        self.body_pos = c64(body_pos)
        lib().orc_set_positions(self.ctx, _dp(self.pos), _dp(self.body_pos))

    def _vec(self, f, x, n_out):
        x = c64(x)
        y = np.zeros(n_out)
        f(self.ctx, _dp(x), _dp(y))
        return y

    def apply_M(self, q):
        return self._vec(lib().orc_apply_M, q, self.N)

    def matvec(self, x):
        return self._vec(lib().orc_matvec, x, self.N + self.B)

    def precondition(self, x):
        return self._vec(lib().orc_precondition, x, self.N + self.B)

    def objective(self, E0):
        return self._vec(lib().orc_objective, E0, self.N + self.B)

    def forces(self, q, E0):
        q, E0 = c64(q), c64(E0)
        f = np.zeros(3 * self.N)
        lib().orc_forces(self.ctx, _dp(q), _dp(E0), _dp(f))
        return f.reshape(-1, 3)

    def gmres(self, b, x0=None, restart=10, maxiter=100, tol=1e-6):
        x = np.zeros(self.N + self.B) if x0 is None else c64(x0).copy()
        b = c64(b)
        resid, true_rel = C.c_double(0), C.c_double(0)
        it = lib().orc_gmres(self.ctx, _dp(x), _dp(b), int(restart), int(maxiter), float(tol),
                             C.byref(resid), C.byref(true_rel))
        return x, it, true_rel.value

    def solve(self, E0, q0=None, phi0=None, restart=10, maxiter=100, tol=1e-6):
        q = np.zeros(self.N) if q0 is None else c64(q0).copy()
        phi = np.zeros(self.B) if phi0 is None else c64(phi0).copy()
        E0 = c64(E0)
        F = np.zeros(3 * self.N)
        true_rel = C.c_double(0)
        it = lib().orc_solve(self.ctx, _dp(E0), _dp(q), _dp(phi), _dp(F), int(restart), int(maxiter), float(tol),
                             C.byref(true_rel))
        return dict(q=q, phi=phi, force=F.reshape(-1, 3), iterations=it, true_rel=true_rel.value)

    def residual(self, q, phi, E0) -> float:
        """True relative residual ||b - A x|| / ||b|| of x = [q; Phi] under this operator."""
        b = self.objective(E0)
        r = b - self.matvec(np.r_[c64(q), c64(phi)])
        return float(np.linalg.norm(r) / np.linalg.norm(b))

    def _body_blocks(self):
        """Inverse saddle-point block of every body with the free-space shell kernel:
        [[-K, 1], [1^T, 0]]^-1 with K(d) = 1/(4 pi d) apart, (4 - d)/(16 pi) for
        overlapping shells (d < 2) and 1/(4 pi) on the diagonal -- each body's own
        isolated-conductor response.  Grouped by body size for batched application."""
        if getattr(self, "_blocks", None) is not None:
            return self._blocks
        body = np.asarray(self.system.body, dtype=np.int64)
        order = np.argsort(body, kind="stable")
        starts = np.searchsorted(body[order], np.arange(self.B + 1))
        by_size = {}
        for b in range(self.B):
            by_size.setdefault(int(starts[b + 1] - starts[b]), []).append(b)
        groups = []
        L = np.asarray(self.system.L, dtype=np.float64)
        for n, bodies in by_size.items():
            idx = np.stack([order[starts[b]:starts[b] + n] for b in bodies])  # (nb, n)
            x = self.pos[idx]
            d = x[:, :, None, :] - x[:, None, :, :]
            d -= L * np.rint(d / L)
            D = np.linalg.norm(d, axis=-1)
            with np.errstate(divide="ignore"):
                K = np.where(D < 2.0, (4.0 - D) / (16.0 * np.pi), 1.0 / (4.0 * np.pi * D))
            K[:, np.arange(n), np.arange(n)] = 1.0 / (4.0 * np.pi)
            A = np.zeros((len(bodies), n + 1, n + 1))
            A[:, :n, :n] = -K
            A[:, :n, n] = 1.0
            A[:, n, :n] = 1.0
            groups.append((idx, np.asarray(bodies), np.linalg.inv(A)))
        self._blocks = groups
        return groups

    def block_precondition(self, v):
        v = c64(v)
        z = np.empty_like(v)
        for idx, bodies, Ainv in self._body_blocks():
            rhs = np.concatenate([v[idx], v[self.N + bodies][:, None]], axis=1)
            sol = np.einsum("bij,bj->bi", Ainv, rhs)
            z[idx] = sol[:, :-1]
            z[self.N + bodies] = sol[:, -1]
        return z

    def solve_tight(self, E0, tol=1e-12, restart=100, maxiter=5000):
        """A tightly converged solution of A x = b under this operator (test reference).

        Right-preconditioned flexible GMRES with the per-body block inverse above and two
        passes of classical Gram-Schmidt, restarted from the true residual b - A x; the
        stopping test is on that true relative residual.  The preconditioner only speeds
        the iteration: the solution is the fixed point of the oracle's own operator
        (ConductorRigid.cu:953-1020), whatever solver reaches it.  Forces follow from the
        oracle's force pass (cu:1256-1278)."""
        E0 = c64(E0)
        b = self.objective(E0)
        n = self.N + self.B
        bnorm = float(np.linalg.norm(b))
        x = np.zeros(n)
        it = 0
        m = int(restart)
        rel = 1.0
        while True:
            r = b - self.matvec(x)
            beta = float(np.linalg.norm(r))
            rel = beta / bnorm if bnorm > 0 else 0.0
            if rel <= tol or it >= maxiter or beta == 0.0:
                break
            V = np.zeros((m + 1, n))
            Z = np.zeros((m, n))
            H = np.zeros((m + 1, m))
            cs, sn = np.zeros(m), np.zeros(m)
            g = np.zeros(m + 1)
            g[0] = beta
            V[0] = r / beta
            k = 0
            for j in range(m):
                Z[j] = self.block_precondition(V[j])
                w = self.matvec(Z[j])
                it += 1
                h = V[: j + 1] @ w
                w -= V[: j + 1].T @ h
                h2 = V[: j + 1] @ w
                w -= V[: j + 1].T @ h2
                h += h2
                hn = float(np.linalg.norm(w))
                H[: j + 1, j] = h
                H[j + 1, j] = hn
                V[j + 1] = w / hn if hn > 0 else 0.0
                for i in range(j):
                    a, c = H[i, j], H[i + 1, j]
                    H[i, j], H[i + 1, j] = cs[i] * a + sn[i] * c, -sn[i] * a + cs[i] * c
                den = float(np.hypot(H[j, j], H[j + 1, j]))
                cs[j], sn[j] = (H[j, j] / den, H[j + 1, j] / den) if den > 0 else (1.0, 0.0)
                H[j, j] = den
                H[j + 1, j] = 0.0
                g[j + 1] = -sn[j] * g[j]
                g[j] = cs[j] * g[j]
                k = j + 1
                if abs(g[j + 1]) <= 0.5 * tol * bnorm or it >= maxiter or hn == 0.0:
                    break
            y = np.linalg.solve(np.triu(H[:k, :k]), g[:k]) if k else np.zeros(0)
            x += Z[:k].T @ y
        q, phi = x[: self.N].copy(), x[self.N:].copy()
        return dict(q=q, phi=phi, force=self.forces(q, E0), iterations=it, true_rel=rel)
