"""Handle-level wrapper of the C ABI over device arrays.

PyTorch provides device memory and streams only; every computation is a call into
libconductor_rigid.so.  Arrays are float64 CUDA tensors; positions are (N, 3).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class Handle:
    """One cr_handle: parameters, tables, mesh, FFT plans and workspaces."""

    def __init__(self, params: _lib.CrParams, L, stream=None):
        import torch

        self.torch = torch
        self.L = np.ascontiguousarray(np.broadcast_to(np.asarray(L, dtype=np.float64), (3,)))
        self.params = params
        self.h = C.c_void_p()
        _lib.check(_lib.lib().cr_create(C.byref(params), _lib.dptr(self.L), C.byref(self.h)), "cr_create")
        if stream is not None:
            self.set_stream(stream)
        self.N = 0
        self.B = 0

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if self.h:
            _lib.lib().cr_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, where, allow=(_lib.CR_OK,)):
        return _lib.check(st, where, self.h, allow)

    def set_stream(self, stream):
        self._check(_lib.lib().cr_set_stream(self.h, C.c_void_p(stream.cuda_stream)), "cr_set_stream")

    def set_tiling(self, tile_edge: int, spread_mode: int = 1):
        self._check(_lib.lib().cr_set_tiling(self.h, int(tile_edge), int(spread_mode)), "cr_set_tiling")

    def autotune(self, pos, body_pos, reps: int = 5) -> dict:
        """Pick the fastest mesh tiling for these positions (leaves them set)."""
        self._pos = self.dev(pos).reshape(-1, 3)
        self._bpos = self.dev(body_pos).reshape(-1, 3)
        t, m, ms = C.c_int(0), C.c_int(0), C.c_float(0)
        self._check(_lib.lib().cr_autotune(self.h, _ptr(self._pos), _ptr(self._bpos), int(reps), C.byref(t),
                                           C.byref(m), C.byref(ms)), "cr_autotune")
        return {"tile_edge": t.value, "spread_mode": m.value, "mesh_ms": ms.value}

    def set_graphs(self, enable: bool):
        self._check(_lib.lib().cr_set_graphs(self.h, int(bool(enable))), "cr_set_graphs")

    def set_realspace(self, flags: int):
        """CR_REALSPACE_ONFLY32 / CR_REALSPACE_ONFLY64: evaluate the real-space kernel values
        of the FP32 / FP64 products on the fly instead of storing them per geometry;
        CR_REALSPACE_STREAM: stream the stored values through shared memory with bulk
        copies (one producer warp per CTA) instead of reading them straight from device
        memory."""
        self._check(_lib.lib().cr_set_realspace(self.h, int(flags)), "cr_set_realspace")

    def set_wait_limit(self, cycles: int = 0, withhold_next: bool = False):
        """Limit of each bounded device wait of the streamed real-space product (SM clock
        cycles; <= 0 restores the default of about a second).  withhold_next: the next
        streamed product issues none of its copies, so its waits run out (a test)."""
        self._check(_lib.lib().cr_set_wait_limit(self.h, C.c_longlong(int(cycles)), int(bool(withhold_next))),
                    "cr_set_wait_limit")

    def set_correction(self, net, weight: float = 1.0):
        """Learned preconditioner correction from `net` (a learned.Network; None removes it)."""
        self._check(_lib.lib().cr_set_correction(self.h, net.h if net is not None else None, C.c_double(weight)),
                    "cr_set_correction")

    def correction_samples(self, max_dirs: int, x, t) -> int:
        """Training rows of the correction from the last solve into x [rows, 48] (int16 BF16
        bits) and t [rows] (float32); returns the number of rows written."""
        rows = C.c_int(0)
        self._check(_lib.lib().cr_correction_samples(self.h, int(max_dirs), _ptr(x), _ptr(t), C.byref(rows)),
                    "cr_correction_samples")
        return rows.value

    def graph_launches(self) -> int:
        v = C.c_longlong(0)
        self._check(_lib.lib().cr_graph_launches(self.h, C.byref(v)), "cr_graph_launches")
        return v.value

    def derived(self) -> _lib.CrDerived:
        d = _lib.CrDerived()
        self._check(_lib.lib().cr_get_derived(self.h, C.byref(d)), "cr_get_derived")
        return d

    def set_field(self, field):
        f = np.ascontiguousarray(field, dtype=np.float64)
        self._check(_lib.lib().cr_set_field(self.h, _lib.dptr(f)), "cr_set_field")

    def set_params(self, params: _lib.CrParams, L=None):
        if L is not None:
            self.L = np.ascontiguousarray(np.broadcast_to(np.asarray(L, dtype=np.float64), (3,)))
        self.params = params
        self._check(_lib.lib().cr_set_params(self.h, C.byref(params), _lib.dptr(self.L)), "cr_set_params")

    def set_topology(self, body, rigid, body_charge):
        body = np.ascontiguousarray(body, dtype=np.uint32)
        rigid = np.ascontiguousarray(rigid, dtype=np.uint8)
        Q = np.ascontiguousarray(body_charge, dtype=np.float64)
        self._check(_lib.lib().cr_set_topology(self.h, len(body), body.ctypes.data_as(C.POINTER(C.c_uint32)),
                                               len(Q), rigid.ctypes.data_as(C.POINTER(C.c_uint8)), _lib.dptr(Q)),
                    "cr_set_topology")
        self.N, self.B = len(body), len(Q)

    # -- device helpers ------------------------------------------------------
    def dev(self, a):
        t = self.torch
        if isinstance(a, t.Tensor):
            return a.to(device="cuda", dtype=t.float64).contiguous()
        return t.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")

    def empty(self, *shape):
        return self.torch.empty(*shape, dtype=self.torch.float64, device="cuda")

    # -- operators -----------------------------------------------------------
    def set_positions(self, pos, body_pos):
        self._pos = self.dev(pos).reshape(-1, 3)
        self._bpos = self.dev(body_pos).reshape(-1, 3)
        self._check(_lib.lib().cr_set_positions(self.h, _ptr(self._pos), _ptr(self._bpos)), "cr_set_positions")

    def apply_operator(self, x, precision=_lib.CR_FP64):
        x = self.dev(x)
        y = self.empty(self.N + self.B)
        self._check(_lib.lib().cr_apply_operator(self.h, _ptr(x), _ptr(y), int(precision)), "cr_apply_operator")
        return y

    def precondition(self, x):
        x = self.dev(x)
        y = self.empty(self.N + self.B)
        self._check(_lib.lib().cr_precondition(self.h, _ptr(x), _ptr(y)), "cr_precondition")
        return y

    def coarse_info(self) -> dict:
        """Coarse level of the two-level preconditioner for the current positions."""
        a, n, m, sp = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
        p = C.c_longlong(0)
        self._check(_lib.lib().cr_coarse_info(self.h, C.byref(a), C.byref(n), C.byref(p), C.byref(m), C.byref(sp)),
                    "cr_coarse_info")
        return {"active": bool(a.value), "n_coarse": n.value, "near_pairs": p.value, "wave_vectors": m.value,
                "sparse": bool(sp.value)}

    def set_coarse(self, max_dense: int = 12288, pcg_iterations: int = 0):
        """Dense limit of the two-level preconditioner's coarse level; above it the level is
        skipped (pcg_iterations 0) or solved in its sparse form by that many CG steps."""
        self._check(_lib.lib().cr_set_coarse(self.h, int(max_dense), int(pcg_iterations)), "cr_set_coarse")

    def objective(self):
        y = self.empty(self.N + self.B)
        self._check(_lib.lib().cr_objective(self.h, _ptr(y)), "cr_objective")
        return y

    def wave_potential(self, q, precision=_lib.CR_FP64):
        q = self.dev(q)
        y = self.empty(self.N)
        self._check(_lib.lib().cr_wave_potential(self.h, _ptr(q), _ptr(y), int(precision)), "cr_wave_potential")
        return y

    def spread(self, q, precision=_lib.CR_FP64):
        q = self.dev(q)
        d = self.derived()
        g = self.empty(d.grid[0] * d.grid[1] * d.grid[2])
        self._check(_lib.lib().cr_spread(self.h, _ptr(q), _ptr(g), int(precision)), "cr_spread")
        return g.reshape(d.grid[0], d.grid[1], d.grid[2])

    def apply_M(self, q, precision=_lib.CR_FP64):
        q = self.dev(q)
        y = self.empty(self.N)
        self._check(_lib.lib().cr_apply_M(self.h, _ptr(q), _ptr(y), int(precision)), "cr_apply_M")
        return y

    def forces(self, q, precision=_lib.CR_FP64):
        q = self.dev(q)
        f = self.empty(self.N, 3)
        self._check(_lib.lib().cr_forces(self.h, _ptr(q), _ptr(f), int(precision)), "cr_forces")
        return f

    def energy(self, q) -> float:
        """1/2 q.(M q) at the current positions (FP64)."""
        q = self.dev(q)
        u = C.c_double(0.0)
        self._check(_lib.lib().cr_energy(self.h, _ptr(q), C.byref(u)), "cr_energy")
        return u.value

    def virial(self, q) -> dict:
        """Virial tensors -dU/de of U = 1/2 q.(M q) at the current positions: real-space and
        wave-space parts as 3x3 arrays, and the wave-space energy."""
        q = self.dev(q)
        v = (C.c_double * 13)()
        self._check(_lib.lib().cr_virial(self.h, _ptr(q), v), "cr_virial")
        a = np.array(v[:])

        def tensor(c):
            return np.array([[c[0], c[1], c[2]], [c[1], c[3], c[4]], [c[2], c[4], c[5]]])

        return {"real": tensor(a[0:6]), "wave": tensor(a[6:12]), "wave_energy": float(a[12])}

    def neighbor_list(self, r_list: float):
        t = self.torch
        count = t.empty(self.N, dtype=t.int32, device="cuda")
        head = t.empty(self.N, dtype=t.int64, device="cuda")
        total = C.c_int64(0)
        self._check(_lib.lib().cr_neighbor_list(self.h, float(r_list), _ptr(count), _ptr(head), None, 0,
                                                C.byref(total)), "cr_neighbor_list")
        lst = t.empty(max(total.value, 1), dtype=t.int32, device="cuda")
        self._check(_lib.lib().cr_neighbor_list(self.h, float(r_list), _ptr(count), _ptr(head), _ptr(lst),
                                                total.value, C.byref(total)), "cr_neighbor_list")
        return count, head, lst[: total.value]

    # -- instrumentation -------------------------------------------------------
    def profile(self, enable: bool = True):
        self._check(_lib.lib().cr_profile(self.h, int(enable)), "cr_profile")

    def profile_read(self) -> dict:
        out = {}
        for k, name in enumerate(_lib.PROFILE_CLASSES):
            n, ms = C.c_int(0), C.c_double(0)
            self._check(_lib.lib().cr_profile_read(self.h, k, C.byref(n), C.byref(ms)), "cr_profile_read")
            out[name] = {"launches": n.value, "ms": ms.value}
        return out

    def geometry_info(self) -> dict:
        g = _lib.CrGeometryInfo()
        self._check(_lib.lib().cr_get_geometry_info(self.h, C.byref(g)), "cr_get_geometry_info")
        return {name: getattr(g, name) for name, _ in g._fields_}

    def counters(self) -> dict:
        a, b = C.c_longlong(0), C.c_longlong(0)
        self._check(_lib.lib().cr_counters(self.h, C.byref(a), C.byref(b)), "cr_counters")
        return {"kernel_launches": a.value, "fft_execs": b.value}

    # -- rigid-body dynamics ---------------------------------------------------
    def body_force_torque(self, pos, body_pos, force):
        """Body forces and torques [B, 3] about the centres from bead forces [N, 3]."""
        pos = self.dev(pos).reshape(-1, 3)
        bpos = self.dev(body_pos).reshape(-1, 3)
        force = self.dev(force).reshape(-1, 3)
        bf = self.empty(self.B, 3)
        bt = self.empty(self.B, 3)
        self._check(_lib.lib().cr_body_force_torque(self.h, _ptr(pos), _ptr(bpos), _ptr(force), _ptr(bf),
                                                    _ptr(bt)), "cr_body_force_torque")
        return bf, bt

    def brownian_step(self, step, radius, force, pos, body_pos, dt=1e-3, kT=1.0, viscosity=1.0, seed=1,
                      repulsion=0.0, contact_gap=0.0):
        """One overdamped rigid-body Brownian step; pos [N, 3] and body_pos [B, 3] (device
        float64 tensors) are moved in place."""
        t = self.torch
        for a in (pos, body_pos):
            if not (isinstance(a, t.Tensor) and a.is_cuda and a.dtype == t.float64 and a.is_contiguous()):
                raise TypeError("pos and body_pos must be contiguous float64 CUDA tensors (moved in place)")
        p = _lib.CrBrownianParams(dt, kT, viscosity, seed, repulsion, contact_gap)
        radius = self.dev(radius)
        force = self.dev(force).reshape(-1, 3)
        self._check(_lib.lib().cr_brownian_step(self.h, C.byref(p), int(step), _ptr(radius), _ptr(force),
                                                _ptr(pos), _ptr(body_pos)), "cr_brownian_step")

    # -- the step --------------------------------------------------------------
    def compute(self, pos, body_pos, q, phi, allow_not_converged=False):
        """Device arrays in, solve + forces; q and phi are updated in place."""
        pos = self.dev(pos).reshape(-1, 3)
        bpos = self.dev(body_pos).reshape(-1, 3)
        force = self.empty(self.N, 3)
        st = _lib.CrSolveStats()
        allow = (_lib.CR_OK, _lib.CR_NOT_CONVERGED) if allow_not_converged else (_lib.CR_OK,)
        self._check(_lib.lib().cr_compute(self.h, _ptr(pos), _ptr(bpos), _ptr(q), _ptr(phi), _ptr(force),
                                          C.byref(st)), "cr_compute", allow)
        return force, st.as_dict()

    def compute_host(self, pos, body_pos, q, phi, force=None, allow_not_converged=False):
        """Host (NumPy) arrays in and out; q and phi are updated in place."""
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        bpos = np.ascontiguousarray(body_pos, dtype=np.float64)
        if force is None:
            force = np.zeros((len(q), 3))
        st = _lib.CrSolveStats()
        allow = (_lib.CR_OK, _lib.CR_NOT_CONVERGED) if allow_not_converged else (_lib.CR_OK,)
        self._check(_lib.lib().cr_compute_host(self.h, _lib.dptr(pos), _lib.dptr(bpos), _lib.dptr(q),
                                               _lib.dptr(phi), _lib.dptr(force), C.byref(st)),
                    "cr_compute_host", allow)
        return force, st.as_dict()
