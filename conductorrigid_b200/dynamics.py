"""Rigid-body Brownian trajectories with one induced-charge solve per step, and the
learned initial guess trained online on the solver's own solutions.

Per step: solve at the current positions (warm start: the previous step's charges and
potentials, as the reference's solve starts from HOOMD's stored charges), then move every
body with the rigid-body Brownian step driven by the electrostatic forces.  With a
LearnedGuess the solve also receives guess directions built from the previous solution
and the motion since: the rotation-transport term and the network's prediction of the
charge change.  The network is trained after each of the first `train_solves` solves on
the change the solver actually produced.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .learned import FEATURES, Network


BEAD_K = 6   # CR_GUESS_BEAD_NEIGHBORS
BODY_K = 8   # CR_GUESS_BODY_NEIGHBORS


def _p(t):
    return C.c_void_p(t.data_ptr())


class LearnedGuess:
    """Guess directions for the next solve from the last solution and the motion since."""

    def __init__(self, handle, radius, *, train_solves=200, passes=4, lr=1e-3, use_network=True,
                 use_transport=True, seed=1):
        import torch

        self.torch = torch
        self.h = handle
        self.radius = handle.dev(radius)
        self.train_solves = train_solves
        self.passes = passes
        self.lr = lr
        self.use_network = use_network
        self.use_transport = use_transport
        self.net = Network(seed=seed) if use_network else None
        self.solves_seen = 0
        self.trained = 0
        self.mu = None
        self.inv_sigma = None
        self.t_scale = None
        N, B = handle.N, handle.B
        dev = "cuda"
        self.bead_nbr = None
        self.body_nbr = torch.empty(B, BODY_K, dtype=torch.int32, device=dev)
        self.feat = torch.empty(N, FEATURES, dtype=torch.float32, device=dev)
        self.xb = torch.empty(N, FEATURES, dtype=torch.int16, device=dev)
        self.transport = torch.empty(N, dtype=torch.float64, device=dev)
        self.target = torch.empty(N, dtype=torch.float32, device=dev)
        self.dirs = torch.zeros(3, N + B, dtype=torch.float64, device=dev)
        self.q_prev = None
        self.losses = []      # training loss (last pass) per training solve
        self.explained = []   # 1 - loss / mean(target^2) per training solve
        self.heldout = []     # the same, on each solve's change before training on it

    def _ck(self, st, where):
        self.h._check(st, where)

    def prepare(self, q_prev, pos_prev, bpos_prev, pos, bpos, phi_prev=None):
        """Features and guess directions for the solve at (pos, bpos); sets them on the handle.

        Directions, in order: the previous solution [q'; Phi'] itself (with the warm start
        x0 = x' the solver's least-squares start can reach both x' and the zero vector, so
        it never starts worse than either), the transport term, the network's prediction
        of the charge change."""
        L = _lib.lib()
        h = self.h.h
        if self.bead_nbr is None:
            self.bead_nbr = self.torch.empty(self.h.N, BEAD_K, dtype=self.torch.int32, device="cuda")
            self._ck(L.cr_bead_neighbors(h, _p(pos_prev), _p(self.bead_nbr)), "cr_bead_neighbors")
        self._ck(L.cr_body_neighbors(h, _p(bpos), _p(self.body_nbr)), "cr_body_neighbors")
        self._ck(L.cr_guess_features(h, _p(self.radius), _p(self.bead_nbr), _p(self.body_nbr), _p(q_prev),
                                     _p(pos_prev), _p(bpos_prev), _p(pos), _p(bpos), _p(self.feat),
                                     _p(self.transport)), "cr_guess_features")
        self.q_prev = q_prev
        k = 0
        if phi_prev is not None:
            self.dirs[k, :self.h.N].copy_(q_prev)
            self.dirs[k, self.h.N:].copy_(phi_prev)
            k += 1
        if self.use_transport:
            self._ck(L.cr_neutral_direction(h, _p(self.transport), 0, C.c_double(1.0), _p(self.dirs[k])),
                     "cr_neutral_direction")
            k += 1
        if self.use_network and self.trained > 0:
            self._pack()
            y = self.net.forward(self.xb)
            self._ck(L.cr_neutral_direction(h, _p(y), 1, C.c_double(self.t_scale), _p(self.dirs[k])),
                     "cr_neutral_direction")
            k += 1
        self._ck(L.cr_set_guess_directions(h, k, _p(self.dirs)), "cr_set_guess_directions")
        return k

    def _pack(self):
        L = _lib.lib()
        self._ck(L.cr_feature_pack(self.h.h, self.h.N, _p(self.feat), _p(self.mu), _p(self.inv_sigma), _p(self.xb)),
                 "cr_feature_pack")

    def learn(self, q):
        """After a solve: score the network on the change the solver produced (held out:
        before training on it), then train on it during the first `train_solves` solves."""
        self.solves_seen += 1
        if not self.use_network or self.q_prev is None:
            return None
        t = self.torch
        L = _lib.lib()
        if self.mu is None:
            sums = t.zeros(2 * FEATURES, dtype=t.float64, device="cuda")
            self._ck(L.cr_feature_stats(self.h.h, self.h.N, _p(self.feat), _p(sums)), "cr_feature_stats")
            s = sums.cpu().numpy()
            n = max(self.h.N, 1)
            mu = s[:FEATURES] / n
            var = np.maximum(s[FEATURES:] / n - mu * mu, 0.0)
            sd = np.sqrt(var)
            self.mu = t.tensor(mu, dtype=t.float32, device="cuda")
            self.inv_sigma = t.tensor(np.where(sd > 1e-12, 1.0 / np.maximum(sd, 1e-300), 0.0), dtype=t.float32,
                                      device="cuda")
            dq = (q - self.q_prev).double()
            self.t_scale = float(max(dq.pow(2).mean().sqrt().item(), 1e-30))
        self._pack()
        self._ck(L.cr_guess_target(self.h.h, _p(q), _p(self.q_prev), C.c_double(self.t_scale), _p(self.target)),
                 "cr_guess_target")
        power = float(self.target.double().pow(2).mean().item())
        if self.trained > 0 and power > 0:
            y = self.net.forward(self.xb).double()
            self.heldout.append(1.0 - float((y - self.target.double()).pow(2).mean().item()) / power)
        if self.trained >= self.train_solves:
            return None
        loss = None
        for _ in range(self.passes):
            loss = self.net.train_step(self.xb, self.target, lr=self.lr)
        self.losses.append(loss)
        self.explained.append(1.0 - loss / power if power > 0 else 0.0)
        self.trained += 1
        return loss


class LearnedCorrection:
    """The learned correction of the preconditioner on one handle, trained online.

    After each of the first `train_solves` solves the handle writes training rows from
    that solve's stored Krylov directions (cr_correction_samples: the features of
    (A z_j, P A z_j) and the targets (z_j - P A z_j) / s), the network is scored on them
    before it sees them (held-out explained fraction) and then trained on them; once
    trained it is switched on with `weight`.  Each solve still decides for itself whether
    to use it (its one-step reduction of the initial residual must beat the plain
    preconditioner's)."""

    def __init__(self, handle, *, train_solves=200, dirs=4, passes=2, lr=1e-3, weight=1.0, seed=2):
        import torch

        self.torch = torch
        self.h = handle
        self.net = Network(seed=seed)
        self.train_solves = train_solves
        self.dirs, self.passes, self.lr, self.weight = dirs, passes, lr, weight
        self.x = torch.empty(dirs * handle.N, FEATURES, dtype=torch.int16, device="cuda")
        self.t = torch.empty(dirs * handle.N, dtype=torch.float32, device="cuda")
        self.trained = 0
        self.losses, self.heldout = [], []
        handle.set_correction(self.net, 0.0)  # weight 0: rows can be drawn, nothing is applied yet

    def learn(self):
        if self.trained >= self.train_solves:
            return None
        rows = self.h.correction_samples(self.dirs, self.x, self.t)
        if rows == 0:
            return None
        x, t = self.x[:rows], self.t[:rows]
        power = float(t.double().pow(2).mean().item())
        if self.trained > 0 and power > 0:
            y = self.net.forward(x).double()
            self.heldout.append(1.0 - float((y - t.double()).pow(2).mean().item()) / power)
        loss = None
        for _ in range(self.passes):
            loss = self.net.train_step(x, t, lr=self.lr)
        self.losses.append(loss)
        self.trained += 1
        if self.trained >= self.train_solves:
            self.h.set_correction(self.net, self.weight)
        return loss


def relax(handle, pos, bpos, radius, steps, *, repulsion=1000.0, contact_gap=0.1, dt=1e-3, kT=1.0, viscosity=1.0,
          seed=1):
    """Brownian steps under the steric repulsion alone (no solves): opens the near-contact
    gaps a random sequential placement leaves.  pos and bpos are moved in place."""
    import torch

    zero = torch.zeros(handle.N, 3, dtype=torch.float64, device="cuda")
    radius = handle.dev(radius)
    for k in range(steps):
        handle.brownian_step(k, radius, zero, pos, bpos, dt=dt, kT=kT, viscosity=viscosity,
                             seed=seed + 0x5EED0000, repulsion=repulsion, contact_gap=contact_gap)


class BrownianRun:
    """One trajectory: solve, then a Brownian step, per call of step()."""

    def __init__(self, handle, system, radius, *, dt=1e-3, kT=1.0, viscosity=1.0, seed=1, guess=None,
                 repulsion=0.0, contact_gap=0.0, relax_steps=0):
        import torch

        self.torch = torch
        self.h = handle
        self.s = system
        self.radius = handle.dev(radius)
        self.dt, self.kT, self.visc, self.seed = dt, kT, viscosity, seed
        self.repulsion, self.contact_gap = repulsion, contact_gap
        self.pos = handle.dev(system.pos).reshape(-1, 3).contiguous()
        self.bpos = handle.dev(system.body_pos).reshape(-1, 3).contiguous()
        self.q = torch.zeros(handle.N, dtype=torch.float64, device="cuda")
        self.phi = torch.zeros(handle.B, dtype=torch.float64, device="cuda")
        self.guess = guess
        self.t = 0
        self.prev = None
        if relax_steps:
            relax(handle, self.pos, self.bpos, radius, relax_steps, repulsion=repulsion or 1000.0,
                  contact_gap=contact_gap or 0.1, dt=dt, kT=kT, viscosity=viscosity, seed=seed)

    def step(self) -> dict:
        e0, e1 = self.torch.cuda.Event(enable_timing=True), self.torch.cuda.Event(enable_timing=True)
        e0.record()
        if self.guess is not None and self.prev is not None:
            self.guess.prepare(self.prev[2], self.prev[0], self.prev[1], self.pos, self.bpos, self.prev[3])
        F, st = self.h.compute(self.pos, self.bpos, self.q, self.phi)
        if self.guess is not None:
            st["train_loss"] = self.guess.learn(self.q)
        e1.record()
        e1.synchronize()
        st["step_ms"] = e0.elapsed_time(e1)  # guess, solve, forces and training (device time)
        self.prev = (self.pos.clone(), self.bpos.clone(), self.q.clone(), self.phi.clone())
        self.h.brownian_step(self.t, self.radius, F, self.pos, self.bpos, dt=self.dt, kT=self.kT,
                             viscosity=self.visc, seed=self.seed, repulsion=self.repulsion,
                             contact_gap=self.contact_gap)
        self.t += 1
        return st


def paired_run(params_plain, params_learned, system, radius, steps, *, train_solves=None, seed=1, dt=1e-3,
               use_network=True, use_transport=True, passes=4, lr=1e-3, repulsion=1000.0, contact_gap=0.1,
               relax_steps=300, mode="lsq", coarse=None, corrected=False, correction_weight=1.0):
    """Solvers on ONE trajectory: the plain solver (warm start from its own previous
    solution) moves the bodies; the learned solver solves the same configurations from its
    own previous solution plus the guess directions; with ``corrected`` a third solver does
    the same as the learned one and also applies the learned preconditioner correction
    (trained online on its own solves during the first ``train_solves``).  Returns per-step
    stats of every arm, the learned guess and the correction (or None).
    ``coarse`` = (max_dense, cg_steps) sets every handle's two-level coarse level."""
    import torch

    from .device import Handle

    stream = torch.cuda.Stream()  # a stream of their own: the solvers capture their Arnoldi steps
    handles = [Handle(params_plain, system.L, stream=stream), Handle(params_learned, system.L, stream=stream)]
    if corrected:
        handles.append(Handle(params_learned, system.L, stream=stream))
    for h in handles:
        h.set_topology(system.body, system.rigid, system.body_charge)
        if coarse is not None:
            h.set_coarse(*coarse)
    with torch.cuda.stream(stream):
        return _paired_loop(handles, system, radius, steps, train_solves, seed, dt, use_network, use_transport,
                            passes, lr, repulsion, contact_gap, relax_steps, mode, correction_weight)


def _paired_loop(handles, system, radius, steps, train_solves, seed, dt, use_network, use_transport, passes, lr,
                 repulsion, contact_gap, relax_steps, mode, correction_weight):
    import torch

    hp, hl = handles[0], handles[1]
    hc = handles[2] if len(handles) > 2 else None
    n_train = train_solves if train_solves is not None else steps
    run = BrownianRun(hp, system, radius, dt=dt, seed=seed, repulsion=repulsion, contact_gap=contact_gap,
                      relax_steps=relax_steps)
    arms = [("learned", hl, LearnedGuess(hl, radius, train_solves=n_train, use_network=use_network,
                                         use_transport=use_transport, passes=passes, lr=lr, seed=seed))]
    corr = None
    if hc is not None:
        arms.append(("corrected", hc, LearnedGuess(hc, radius, train_solves=n_train, use_network=use_network,
                                                   use_transport=use_transport, passes=passes, lr=lr, seed=seed)))
        corr = LearnedCorrection(hc, train_solves=n_train, lr=lr, weight=correction_weight, seed=seed + 1)
    state = {name: [torch.zeros(h.N, dtype=torch.float64, device="cuda"),
                    torch.zeros(h.B, dtype=torch.float64, device="cuda"), None] for name, h, _ in arms}
    out = []
    for k in range(steps):
        pos, bpos = run.pos.clone(), run.bpos.clone()
        rec = {}
        for name, h, guess in arms:
            q, ph, prev = state[name]
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            if prev is not None:
                nd = guess.prepare(prev[2], prev[0], prev[1], pos, bpos, None if mode == "add" else prev[3])
                if mode == "add":
                    # unit-weight corrections on top of the warm start
                    for j in range(nd):
                        q += guess.dirs[j, :h.N]
                    _lib.lib().cr_set_guess_directions(h.h, 0, None)
            _, st = h.compute(pos, bpos, q, ph)
            st["train_loss"] = guess.learn(q)
            if name == "corrected":
                st["correction_loss"] = corr.learn()
            e1.record()
            e1.synchronize()
            st["step_ms"] = e0.elapsed_time(e1)
            state[name][2] = (pos, bpos, q.clone(), ph.clone())
            rec[name] = st
        rec["plain"] = run.step()
        out.append(rec)
    for h in handles:
        h.close()
    return out, arms[0][2], corr
