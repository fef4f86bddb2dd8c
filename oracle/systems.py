"""Benchmark systems built on the oracle side (TEST INFRASTRUCTURE).

The CPU baseline and the reference-method arm of the benchmark build their inputs
here, through the oracle library only, so that they never load the CUDA product.
The workloads are the product's (same names, seeds and parameters); the primitives
(icosphere, SplitMix64 uniforms, random sequential addition) are the oracle's own
restatement in cr_systems.cc, and tests/test_oracle_systems.py checks that both
generators give identical arrays.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _dp, lib

XI_DEFAULT = math.sqrt(-math.log(1e-5)) / 4.0


@dataclass
class System:
    L: np.ndarray
    pos: np.ndarray
    body: np.ndarray
    rigid: np.ndarray
    body_charge: np.ndarray
    body_pos: np.ndarray
    radius: np.ndarray
    field: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def n_beads(self) -> int:
        return int(self.pos.shape[0])

    @property
    def n_bodies(self) -> int:
        return int(self.rigid.shape[0])


def _sigs():
    L = lib()
    if not getattr(L, "_systems_sigs", False):
        L.orc_icosphere_count.argtypes, L.orc_icosphere_count.restype = [C.c_int], C.c_int
        L.orc_icosphere.argtypes, L.orc_icosphere.restype = [C.c_int, C.POINTER(C.c_double)], C.c_int
        L.orc_uniform.argtypes, L.orc_uniform.restype = [C.c_uint64, C.c_int64, C.POINTER(C.c_double)], C.c_int
        L.orc_place_spheres.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_uint64,
                                        C.c_int64, C.POINTER(C.c_double)]
        L.orc_place_spheres.restype = C.c_int
        L._systems_sigs = True
    return L


def icosphere(level: int) -> np.ndarray:
    L = _sigs()
    n = L.orc_icosphere_count(int(level))
    if n < 0:
        raise ValueError(f"unsupported icosphere level {level}")
    v = np.zeros(3 * n)
    if L.orc_icosphere(int(level), _dp(v)) != 0:
        raise RuntimeError("orc_icosphere failed")
    return v.reshape(n, 3)


def uniform(seed: int, n: int) -> np.ndarray:
    out = np.zeros(int(n))
    if n and _sigs().orc_uniform(C.c_uint64(seed), int(n), _dp(out)) != 0:
        raise RuntimeError("orc_uniform failed")
    return out


def place_spheres(radii, L, seed: int, max_attempts: int = 200_000_000) -> np.ndarray:
    radii = np.ascontiguousarray(radii, dtype=np.float64)
    Lv = np.ascontiguousarray(np.broadcast_to(np.asarray(L, dtype=np.float64), (3,)))
    out = np.zeros(3 * len(radii))
    if _sigs().orc_place_spheres(len(radii), _dp(radii), _dp(Lv), C.c_uint64(seed), int(max_attempts),
                                 _dp(out)) != 0:
        raise RuntimeError("orc_place_spheres: no room for the spheres within the attempt limit")
    return out.reshape(-1, 3)


def spheres(radii, levels, phi: float, E0=(0.0, 0.0, 1.0), charges=None, seed: int = 1) -> System:
    radii = np.asarray(radii, dtype=np.float64)
    levels = np.broadcast_to(np.asarray(levels, dtype=np.int64), radii.shape)
    B = len(radii)
    Ledge = (float(np.sum(4.0 / 3.0 * np.pi * radii ** 3)) / phi) ** (1.0 / 3.0)
    L = np.array([Ledge] * 3)
    centres = place_spheres(radii, L, seed)
    verts = {int(lv): icosphere(int(lv)) for lv in np.unique(levels)}
    pos = np.concatenate([centres[b] + radii[b] * verts[int(levels[b])] for b in range(B)])
    pos = pos - L * np.floor((pos + 0.5 * L) / L)
    body = np.concatenate([np.full(len(verts[int(levels[b])]), b, dtype=np.uint32) for b in range(B)])
    Q = np.zeros(B) if charges is None else np.asarray(charges, dtype=np.float64)
    return System(L=L, pos=np.ascontiguousarray(pos), body=np.ascontiguousarray(body),
                  rigid=np.ones(B, dtype=np.uint8), body_charge=np.ascontiguousarray(Q),
                  body_pos=np.ascontiguousarray(centres), radius=radii, field=np.asarray(E0, dtype=np.float64),
                  meta={"phi": phi, "seed": seed})


def _params(grid, support, **kw) -> dict:
    p = dict(xi=XI_DEFAULT, errortol=1e-5, rcut=4.0, grid=grid, support=support, gmres_tol=1e-6)
    p.update(kw)
    return p


def workload(name: str, seed: int = 1, scale: float = 1.0):
    """(system, params) of the named benchmark workload; ``scale`` < 1 shrinks the body
    count at the same volume fraction."""
    if name == "plain_small":
        nb = max(1, int(round(100 * scale)))
        return spheres(np.ones(nb), 1, 0.10, seed=seed), _params(64, 9)
    if name == "precision_162k":
        nb = max(1, int(round(1000 * scale)))
        return spheres(np.ones(nb), 2, 0.30, seed=seed), _params(128, 11)
    if name == "polydisperse_204k":
        nh = max(1, int(round(1000 * scale)))
        radii = np.concatenate([np.ones(nh), 2.0 * np.ones(nh)])
        levels = np.concatenate([np.ones(nh, dtype=int), 2 * np.ones(nh, dtype=int)])
        signs = np.concatenate([np.ones(nh), -np.ones(nh)])
        perm = np.argsort(uniform(seed + 7919, 2 * nh), kind="stable")
        return spheres(radii, levels, 0.25, (0.3, 0.0, 1.0), charges=signs[perm], seed=seed), _params(256, 11)
    raise KeyError(name)
