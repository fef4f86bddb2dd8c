"""Python force compute with the reference plugin's surface (pymodule/compute.py).

``ConductorRigid(group, body, charge, field=[0,0,0], xi=0.5, errortol=1e-3,
fileprefix="", period=0)`` computes the forces on charged rigid conductors in an
external field, as the reference's class does for a HOOMD-blue system
(pymodule/compute.py:16-64).  HOOMD is not part of this package, so the system is
passed explicitly as a keyword: any object with ``pos`` (N, 3), ``body_pos`` (B, 3),
``rigid`` (B,) and ``L`` (3,) arrays, such as ``systems.ConductorSystem``.  The group
must be all beads in index order (the reference's GMRES vector mixes group and global
indices, ConductorRigid.cu:169 and :994, which agree only for that group).  Extra
keyword options that the reference hard-codes or derives: ``grid``, ``support``,
``rcut``, ``gmres_tol``, ``restart``, ``maxiter``, ``precision`` ("fp64", "mixed"),
``precond`` ("diagonal", "conductor", "two_level").
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib


class _SystemArrays:
    """Contiguous float64 / uint8 views the C++ object points into."""

    def __init__(self, system):
        self.pos = np.ascontiguousarray(system.pos, dtype=np.float64)
        self.body_pos = np.ascontiguousarray(system.body_pos, dtype=np.float64)
        self.rigid = np.ascontiguousarray(system.rigid, dtype=np.uint8)
        self.L = np.ascontiguousarray(np.broadcast_to(np.asarray(system.L, dtype=np.float64), (3,)))
        self.charge = np.zeros(self.pos.shape[0], dtype=np.float64)


class ConductorRigid:
    """Forces on charged rigid-body conductors in an external field."""

    def __init__(self, group, body, charge, field=[0.0, 0.0, 0.0], xi=0.5, errortol=1e-3, fileprefix="", period=0,
                 *, system, t0=0, **options):
        # set the cutoff radius (compute.py:27)
        self.rcut = math.sqrt(-math.log(errortol)) / xi
        self.enabled = True
        import torch

        # the reference refuses to run without CUDA (compute.py:33-35)
        if not torch.cuda.is_available():
            raise RuntimeError("Error creating ConductorRigid")
        n = int(np.asarray(system.pos).shape[0])
        if group not in (None, "all") and not np.array_equal(np.asarray(group), np.arange(n)):
            raise ValueError("ConductorRigid supports the group of all beads in index order")
        from . import _ConductorRigid  # noqa: PLC0415  (built by conductorrigid_b200.build)

        opts = dict(options)
        if "precision" in opts and isinstance(opts["precision"], str):
            opts["precision"] = _lib.PRECISIONS[opts["precision"]]
        if "precond" in opts and isinstance(opts["precond"], str):
            opts["precond"] = _lib.PRECONDITIONERS[opts["precond"]]
        self._arrays = _SystemArrays(system)
        self._t0 = int(t0)
        self.cpp_force = _ConductorRigid.ConductorRigid(self._arrays, [int(b) for b in body],
                                                        [float(q) for q in charge], list(field), float(xi),
                                                        float(errortol), str(fileprefix), int(period), self._t0, opts)
        # set parameters for the force (compute.py:51)
        self.cpp_force.SetParams()

    # Update only the external field (compute.py:54-55)
    def update_field(self, field):
        self.cpp_force.UpdateField(list(field))

    # Update simulation parameters (compute.py:58-60)
    def update_parameters(self, field, fileprefix, period):
        self.cpp_force.UpdateParams(list(field), str(fileprefix), int(period), self._t0)
        self.cpp_force.SetParams()

    # The integrator calls update_coeffs but there are no coefficients (compute.py:63-64)
    def update_coeffs(self):
        pass

    def compute(self, timestep: int = 0):
        """One step: solve for charges and body potentials, then bead forces."""
        self.cpp_force.computeForces(int(timestep))
        return self.cpp_force.forces

    def set_positions(self, pos, body_pos=None):
        """Move the beads (and body centres) in place for the next step."""
        self._arrays.pos[...] = pos
        if body_pos is not None:
            self._arrays.body_pos[...] = body_pos

    @property
    def charges(self) -> np.ndarray:
        return self._arrays.charge

    @property
    def potentials(self) -> np.ndarray:
        return self.cpp_force.potentials

    @property
    def forces(self) -> np.ndarray:
        return self.cpp_force.forces

    @property
    def stats(self) -> dict:
        return self.cpp_force.stats
