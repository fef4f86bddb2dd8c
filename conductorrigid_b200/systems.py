"""Synthetic conductor systems of the benchmark workloads.

Each conductor is a sphere of radius ``a`` carrying beads at the vertices of an
icosphere (level 1: 42 beads, level 2: 162 beads) at radius ``a``; every bead is a
unit-radius charged shell, as in the reference kernel.  Sphere centres are placed by
random sequential addition in a periodic cubic box at the requested volume fraction,
with a SplitMix64 generator so that a seed fixes the system on every machine.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib

#: Ewald split used by every workload: real-space truncation 1e-5 at cutoff 4
XI_DEFAULT = math.sqrt(-math.log(1e-5)) / 4.0


@dataclass
class ConductorSystem:
    L: np.ndarray            # (3,) box edges
    pos: np.ndarray          # (N, 3) bead positions in [-L/2, L/2)
    body: np.ndarray         # (N,) uint32 body tag of each bead
    rigid: np.ndarray        # (B,) uint8, 1 for rigid bodies
    body_charge: np.ndarray  # (B,) total charge of each body
    body_pos: np.ndarray     # (B, 3) body centres
    radius: np.ndarray       # (B,) body radii
    field: np.ndarray        # (3,) external field
    meta: dict = field(default_factory=dict)

    @property
    def n_beads(self) -> int:
        return int(self.pos.shape[0])

    @property
    def n_bodies(self) -> int:
        return int(self.rigid.shape[0])


def icosphere(level: int) -> np.ndarray:
    n = _lib.lib().cr_util_icosphere_count(int(level))
    if n < 0:
        raise ValueError(f"unsupported icosphere level {level}")
    v = np.zeros(3 * n)
    _lib.check(_lib.lib().cr_util_icosphere(int(level), _lib.dptr(v)), "cr_util_icosphere")
    return v.reshape(n, 3)


def uniform(seed: int, n: int) -> np.ndarray:
    out = np.zeros(int(n))
    if n:
        _lib.check(_lib.lib().cr_util_uniform(C.c_uint64(seed), int(n), _lib.dptr(out)), "cr_util_uniform")
    return out


def place_spheres(radii: np.ndarray, L, seed: int, max_attempts: int = 200_000_000) -> np.ndarray:
    radii = np.ascontiguousarray(radii, dtype=np.float64)
    Lv = np.ascontiguousarray(np.broadcast_to(np.asarray(L, dtype=np.float64), (3,)))
    out = np.zeros(3 * len(radii))
    st = _lib.lib().cr_util_place_spheres(len(radii), _lib.dptr(radii), _lib.dptr(Lv), C.c_uint64(seed),
                                          int(max_attempts), _lib.dptr(out))
    _lib.check(st, "cr_util_place_spheres")
    return out.reshape(-1, 3)


def wrap(x: np.ndarray, L: np.ndarray) -> np.ndarray:
    return x - L * np.floor((x + 0.5 * L) / L)


def spheres(radii, levels, phi: float, field=(0.0, 0.0, 1.0), charges=None, seed: int = 1) -> ConductorSystem:
    """Conducting spheres of the given radii / icosphere levels at volume fraction phi."""
    radii = np.asarray(radii, dtype=np.float64)
    levels = np.broadcast_to(np.asarray(levels, dtype=np.int64), radii.shape)
    B = len(radii)
    vol = float(np.sum(4.0 / 3.0 * np.pi * radii ** 3))
    Ledge = (vol / phi) ** (1.0 / 3.0)
    L = np.array([Ledge] * 3)
    centres = place_spheres(radii, L, seed)
    verts = {lvl: icosphere(int(lvl)) for lvl in np.unique(levels)}
    pos, body = [], []
    for b in range(B):
        v = verts[int(levels[b])]
        pos.append(centres[b] + radii[b] * v)
        body.append(np.full(len(v), b, dtype=np.uint32))
    pos = wrap(np.concatenate(pos), L) if B else np.zeros((0, 3))
    body = np.concatenate(body) if B else np.zeros(0, dtype=np.uint32)
    q = np.zeros(B) if charges is None else np.asarray(charges, dtype=np.float64)
    return ConductorSystem(
        L=L,
        pos=np.ascontiguousarray(pos),
        body=np.ascontiguousarray(body),
        rigid=np.ones(B, dtype=np.uint8),
        body_charge=np.ascontiguousarray(q),
        body_pos=np.ascontiguousarray(centres),
        radius=radii,
        field=np.asarray(field, dtype=np.float64),
        meta={"phi": phi, "seed": seed},
    )


@dataclass
class Workload:
    name: str
    system: ConductorSystem
    params: dict


def _base_params(grid, support, **kw) -> dict:
    p = dict(xi=XI_DEFAULT, errortol=1e-5, rcut=4.0, grid=grid, support=support, gmres_tol=1e-6,
             restart=10, maxiter=1000)
    p.update(kw)
    return p


def workload(name: str, seed: int = 1, scale: float = 1.0) -> Workload:
    """The named workloads.  ``scale`` < 1 shrinks the body count (tests)."""
    if name == "plain_small":
        # 100 spheres a=1, 42 beads, phi 0.10, E0 (0,0,1), mesh 64^3, P=9, FP64
        nb = max(1, int(round(100 * scale)))
        s = spheres(np.ones(nb), 1, 0.10, (0.0, 0.0, 1.0), seed=seed)
        return Workload(name, s, _base_params(64, 9, precision="fp64"))
    if name == "precision_162k":
        # 1000 spheres a=1, 162 beads, phi 0.30, mesh 128^3, P=11
        nb = max(1, int(round(1000 * scale)))
        s = spheres(np.ones(nb), 2, 0.30, (0.0, 0.0, 1.0), seed=seed)
        return Workload(name, s, _base_params(128, 11, precision="mixed"))
    if name == "dynamics_420k":
        # 10000 spheres a=1, 42 beads, phi 0.35, mesh 256^3, P=9
        nb = max(1, int(round(10000 * scale)))
        s = spheres(np.ones(nb), 1, 0.35, (0.0, 0.0, 1.0), seed=seed)
        return Workload(name, s, _base_params(256, 9, precision="mixed"))
    if name == "polydisperse_204k":
        # 1000 a=1 (42 beads) + 1000 a=2 (162 beads), Q = +-1 summing to zero,
        # phi 0.25, E0 (0.3, 0, 1), mesh 256^3, P=11, cutoff 4
        nh = max(1, int(round(1000 * scale)))
        radii = np.concatenate([np.ones(nh), 2.0 * np.ones(nh)])
        levels = np.concatenate([np.ones(nh, dtype=int), 2 * np.ones(nh, dtype=int)])
        signs = np.concatenate([np.ones(nh), -np.ones(nh)])
        perm = np.argsort(uniform(seed + 7919, 2 * nh), kind="stable")
        s = spheres(radii, levels, 0.25, (0.3, 0.0, 1.0), charges=signs[perm], seed=seed)
        return Workload(name, s, _base_params(256, 11, precision="mixed"))
    raise KeyError(name)


def replica_specs(n_replicas: int = 256, seed: int = 1):
    """Batched uneven replicas: N_body ~ U[20, 400], phi ~ U[0.05, 0.35], field
    direction uniform on the sphere with magnitude 1, zero body charges; mesh
    2 points per unit length rounded up to a 5-smooth size (at most 128), P=9."""
    u = uniform(seed + 104729, 4 * n_replicas).reshape(n_replicas, 4)
    specs = []
    for r in range(n_replicas):
        nb = 20 + int(u[r, 0] * 381)
        phi = 0.05 + 0.30 * u[r, 1]
        cz = 2.0 * u[r, 2] - 1.0
        ph = 2.0 * np.pi * u[r, 3]
        sz = math.sqrt(max(0.0, 1.0 - cz * cz))
        specs.append(dict(n_bodies=nb, phi=phi, field=(sz * math.cos(ph), sz * math.sin(ph), cz), seed=seed + r))
    return specs


def smooth_at_least(n: int, cap: int = 128) -> int:
    best = None
    for a in range(13):
        for b in range(8):
            for c in range(6):
                m = 2 ** a * 3 ** b * 5 ** c
                if m >= n and (best is None or m < best):
                    best = m
    return min(best, cap)
