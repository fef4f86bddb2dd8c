"""Many independent periodic systems of uneven size, solved side by side.

Each replica is a full system with its own handle: box, mesh (2 nodes per unit length,
rounded up to a 5-smooth size of at most 128), Ewald parameter and topology.  The
real-space sum takes one image per pair, as the reference's does, so it needs
rc <= L/2; for boxes smaller than 2 rc the replica's Ewald parameter is raised to
xi = sqrt(-ln tol)/rc with rc = L/2, which keeps the real-space truncation error at the
tolerance and moves the rest of the sum to the mesh.

solve_lockstep() runs all replicas through a lockstep batch (cr_batch_create /
cr_batch_solve): every unconverged replica takes one Arnoldi step per round and each stage
of the step is one kernel launch over all replicas.  solve_batched() runs them through
cr_batch_compute (concurrent streams, each Arnoldi step a captured graph);
solve_looped() solves them one after another through cr_compute, the single-system path.  With autotune=True every replica's mesh tiling is
chosen by cr_autotune at construction (each system timed alone); tune_batch() instead
chooses the tiling policy by the batch's own throughput.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib, systems
from .device import Handle


def replica_params(system, tol=1e-5, support=9, gmres_tol=1e-6, restart=50, maxiter=4000, precision="mixed",
                   precond="conductor", rc_max=4.0):
    L = float(min(system.L))
    rc = min(rc_max, 0.5 * L * (1.0 - 1e-12))
    xi = math.sqrt(-math.log(tol)) / rc
    grid = tuple(systems.smooth_at_least(int(math.ceil(2.0 * Ld))) for Ld in system.L)
    return _lib.make_params(field=tuple(system.field), xi=xi, errortol=tol, grid=grid, support=support, rcut=rc,
                            gmres_tol=gmres_tol, restart=restart, maxiter=maxiter, precision=precision,
                            precond=precond)


class Replicas:
    def __init__(self, specs, autotune=False, **param_kw):
        import torch

        self.torch = torch
        self.systems = []
        self.handles = []
        self.arrays = []
        for sp in specs:
            s = systems.spheres(np.ones(sp["n_bodies"]), 1, sp["phi"], sp["field"], seed=sp["seed"])
            h = Handle(replica_params(s, **param_kw), s.L)
            h.set_topology(s.body, s.rigid, s.body_charge)
            pos = h.dev(s.pos).reshape(-1, 3).contiguous()
            bpos = h.dev(s.body_pos).reshape(-1, 3).contiguous()
            q = torch.zeros(s.n_beads, dtype=torch.float64, device="cuda")
            phi = torch.zeros(s.n_bodies, dtype=torch.float64, device="cuda")
            force = torch.zeros(s.n_beads, 3, dtype=torch.float64, device="cuda")
            self.systems.append(s)
            self.handles.append(h)
            self.arrays.append((pos, bpos, q, phi, force))
        self.n = len(self.handles)
        self.tilings = [h.autotune(a[0], a[1], reps=3) for h, a in zip(self.handles, self.arrays)] if autotune else []
        self.n_charges = sum(s.n_beads for s in self.systems)

    def reset(self):
        for (_, _, q, phi, _) in self.arrays:
            q.zero_()
            phi.zero_()

    def warm(self):
        """One solve per replica: allocates every handle's per-solve buffers."""
        self.reset()
        self.solve_looped()
        self.reset()

    def solve_looped(self):
        stats = []
        for h, (pos, bpos, q, phi, force) in zip(self.handles, self.arrays):
            st = _lib.CrSolveStats()
            code = _lib.lib().cr_compute(h.h, C.c_void_p(pos.data_ptr()), C.c_void_p(bpos.data_ptr()),
                                         C.c_void_p(q.data_ptr()), C.c_void_p(phi.data_ptr()),
                                         C.c_void_p(force.data_ptr()), C.byref(st))
            h._check(code, "cr_compute")
            stats.append(st.as_dict())
        self.torch.cuda.synchronize()
        return stats

    def solve_batched(self, n_threads=16):
        n = self.n
        P = C.c_void_p * n
        hs = P(*[h.h.value for h in self.handles])
        cols = [P(*[a[k].data_ptr() for a in self.arrays]) for k in range(5)]
        st = (_lib.CrSolveStats * n)()
        status = (C.c_int * n)()
        code = _lib.lib().cr_batch_compute(n, hs, *cols, st, status, int(n_threads))
        if code != _lib.CR_OK:
            bad = [i for i in range(n) if status[i] != _lib.CR_OK]
            raise _lib.CrError(code, "cr_batch_compute", f"replicas {bad[:8]} failed")
        return [st[i].as_dict() for i in range(n)]

    def _columns(self):
        n = self.n
        P = C.c_void_p * n
        return [P(*[a[k].data_ptr() for a in self.arrays]) for k in range(5)]

    def _lockstep_tiling(self):
        """The lockstep batch's tiling (8^3 tiles, register-column spreading) on every handle,
        set again only after tune_batch or set_tilings changed it."""
        if not getattr(self, "_default_tiling", False):
            for h in self.handles:
                h.set_tiling(8, 0)
            self._default_tiling = True

    def make_lockstep(self):
        """The lockstep batch over these replicas' handles (8^3 register-column tiling)."""
        self._lockstep_tiling()
        if getattr(self, "_lockstep", None) is not None:
            return self._lockstep
        n = self.n
        hs = (C.c_void_p * n)(*[h.h.value for h in self.handles])
        out = C.c_void_p()
        code = _lib.lib().cr_batch_create(n, hs, C.byref(out))
        if code != _lib.CR_OK:
            msg = (_lib.lib().cr_batch_last_error(None) or b"").decode()
            raise _lib.CrError(code, "cr_batch_create", msg)
        self._lockstep = out
        return out

    def solve_lockstep(self, n_threads=16):
        """All replicas in one lockstep batch: per-geometry set-up and forces per replica on
        n_threads host threads, the iterations one launch per stage over every replica."""
        bt = self.make_lockstep()
        n = self.n
        st = (_lib.CrSolveStats * n)()
        status = (C.c_int * n)()
        code = _lib.lib().cr_batch_solve(bt, *self._columns(), st, status, int(n_threads))
        if code != _lib.CR_OK:
            bad = [i for i in range(n) if status[i] != _lib.CR_OK]
            msg = (_lib.lib().cr_batch_last_error(bt) or b"").decode()
            raise _lib.CrError(code, "cr_batch_solve", f"{msg}; replicas {bad[:8]} failed")
        return [st[i].as_dict() for i in range(n)]

    def lockstep_counters(self):
        """(batched kernel launches, batched transforms, lockstep rounds) so far."""
        a, b, c = C.c_longlong(), C.c_longlong(), C.c_longlong()
        _lib.lib().cr_batch_counters(self.make_lockstep(), C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def lockstep_phases(self):
        """Last lockstep solve: ms until the first replica joined the rounds, ms of the
        rounds from then on (device), ms of the whole call (host)."""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        _lib.lib().cr_batch_phase_ms(self.make_lockstep(), C.byref(a), C.byref(b), C.byref(c))
        return {"first_join": a.value, "rounds": b.value, "total": c.value}

    def set_tilings(self, tilings):
        self._default_tiling = False
        for h, t in zip(self.handles, tilings):
            h.set_tiling(t["tile_edge"], t["spread_mode"])

    def tune_batch(self, n_threads=16, policies=((8, 0), (4, 1), (6, 1), "isolated")):
        """Pick the mesh tiling by the throughput of the batch itself.  Per-replica tuning
        (cr_autotune) times each system alone, where small tiles win by occupying more of
        the GPU; in a batch the GPU is already full and the extra halo work of small tiles
        costs throughput, so the policy is chosen by timing one batched solve under each.
        Returns {policy: solves/s}; the fastest policy stays set."""
        import time

        if "isolated" in policies and not self.tilings:
            self.tilings = [h.autotune(a[0], a[1], reps=3) for h, a in zip(self.handles, self.arrays)]
        rates = {}
        self._default_tiling = False
        for pol in policies:
            if pol == "isolated":
                self.set_tilings(self.tilings)
            else:
                for h in self.handles:
                    h.set_tiling(*pol)
            self.warm()
            self.solve_batched(n_threads)  # captures this policy's graphs
            self.reset()
            self.torch.cuda.synchronize()
            t0 = time.perf_counter()
            self.solve_batched(n_threads)
            self.torch.cuda.synchronize()
            rates[str(pol)] = self.n / (time.perf_counter() - t0)
            self.reset()
        best = max(policies, key=lambda p: rates[str(p)])
        if best == "isolated":
            self.set_tilings(self.tilings)
        else:
            for h in self.handles:
                h.set_tiling(*best)
        self.best_policy = str(best)
        self.warm()
        return rates

    def close(self):
        if getattr(self, "_lockstep", None) is not None:
            _lib.lib().cr_batch_destroy(self._lockstep)
            self._lockstep = None
        for h in self.handles:
            h.close()
        self.handles = []
