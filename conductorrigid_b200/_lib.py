"""ctypes binding of the C ABI in include/conductor_rigid.h.

The shared library ``libconductor_rigid.so`` is built in-tree by
``conductorrigid_b200.build``.  There is no fallback: if the library is missing
every entry point raises, so a GPU run can never silently use something else.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libconductor_rigid.so"

CR_OK = 0
CR_NOT_CONVERGED = 1
CR_BAD_PARAM = 2
CR_CUDA_ERROR = 3
CR_TIMEOUT = 4
CR_OUT_OF_MEMORY = 5
CR_GRID_TOO_LARGE = 6
CR_NOT_READY = 7
CR_NUMERICAL = 8

CR_FP64 = 0
CR_MIXED = 1
CR_FP32 = 2

PRECISIONS = {"fp64": CR_FP64, "mixed": CR_MIXED, "fp32": CR_FP32}

CR_REALSPACE_ONFLY32 = 1
CR_REALSPACE_ONFLY64 = 2
CR_REALSPACE_STREAM = 4
CR_REALSPACE_SERIAL = 8

CR_PRECOND_DIAGONAL = 0
CR_PRECOND_CONDUCTOR = 1
CR_PRECOND_TWO_LEVEL = 2
PRECONDITIONERS = {"diagonal": CR_PRECOND_DIAGONAL, "conductor": CR_PRECOND_CONDUCTOR,
                   "two_level": CR_PRECOND_TWO_LEVEL}

#: kernel classes of cr_profile_read
PROFILE_CLASSES = ["spread", "fft", "scale", "contract", "real_space", "contract_force", "real_space_force",
                   "krylov", "body", "geometry", "precondition", "coarse"]


class CrParams(C.Structure):
    _fields_ = [
        ("field", C.c_double * 3),
        ("xi", C.c_double),
        ("errortol", C.c_double),
        ("grid", C.c_int * 3),
        ("support", C.c_int),
        ("rcut", C.c_double),
        ("gmres_tol", C.c_double),
        ("restart", C.c_int),
        ("maxiter", C.c_int),
        ("precision", C.c_int),
        ("learned", C.c_int),
        ("precond", C.c_int),
    ]


class CrDerived(C.Structure):
    _fields_ = [
        ("grid", C.c_int * 3),
        ("support", C.c_int),
        ("support_unclamped", C.c_int),
        ("h", C.c_double * 3),
        ("eta", C.c_double * 3),
        ("rcut", C.c_double),
        ("kcut", C.c_double),
        ("n_table", C.c_int),
        ("dr", C.c_double),
        ("selfcoeff", C.c_double),
        ("xiterm", C.c_double),
        ("prefac", C.c_double),
        ("quadW", C.c_double),
    ]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class CrSolveStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int),
        ("restarts", C.c_int),
        ("refinements", C.c_int),
        ("matvecs_fp64", C.c_int),
        ("matvecs_fp32", C.c_int),
        ("converged", C.c_int),
        ("used_learned_guess", C.c_int),
        ("initial_residual", C.c_double),
        ("final_residual", C.c_double),
        ("solve_ms", C.c_double),
        ("learned_residual", C.c_double),
        ("used_learned_correction", C.c_int),
        ("correction_reduction", C.c_double * 2),
    ]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class CrGeometryInfo(C.Structure):
    _fields_ = [
        ("real_space_pairs", C.c_int64),
        ("tile_edge", C.c_int),
        ("n_tiles", C.c_int),
        ("n_beads", C.c_int),
        ("n_bodies", C.c_int),
        ("cluster_pairs", C.c_int64),
        ("stored_values", C.c_int64),
    ]


class CrBrownianParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("kT", C.c_double), ("viscosity", C.c_double), ("seed", C.c_uint64),
                ("repulsion", C.c_double), ("contact_gap", C.c_double)]


class CrError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str = ""):
        self.status = status
        super().__init__(f"{where}: {status_string(status)} ({status}){': ' + msg if msg else ''}")


_lib = None

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I = C.c_int
_SIGS = {
    "cr_abi_version": ([], _I),
    "cr_status_string": ([_I], C.c_char_p),
    "cr_last_error": ([_P], C.c_char_p),
    "cr_derive_params": ([C.POINTER(CrParams), _D, C.POINTER(CrDerived)], _I),
    "cr_build_tables": ([C.POINTER(CrDerived), C.c_double, _D, _D], _I),
    "cr_create": ([C.POINTER(CrParams), _D, C.POINTER(_P)], _I),
    "cr_destroy": ([_P], _I),
    "cr_get_derived": ([_P, C.POINTER(CrDerived)], _I),
    "cr_set_field": ([_P, _D], _I),
    "cr_set_params": ([_P, C.POINTER(CrParams), _D], _I),
    "cr_set_topology": ([_P, _I, C.POINTER(C.c_uint32), _I, C.POINTER(C.c_uint8), _D], _I),
    "cr_set_stream": ([_P, _P], _I),
    "cr_set_graphs": ([_P, _I], _I),
    "cr_set_realspace": ([_P, _I], _I),
    "cr_set_wait_limit": ([_P, C.c_longlong, _I], _I),
    "cr_set_correction": ([_P, _P, C.c_double], _I),
    "cr_correction_samples": ([_P, _I, _P, _P, C.POINTER(C.c_int)], _I),
    "cr_set_tiling": ([_P, _I, _I], _I),
    "cr_autotune": ([_P, _P, _P, _I, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float)], _I),
    "cr_graph_launches": ([_P, C.POINTER(C.c_longlong)], _I),
    "cr_compute": ([_P, _P, _P, _P, _P, _P, C.POINTER(CrSolveStats)], _I),
    "cr_compute_host": ([_P, _D, _D, _D, _D, _D, C.POINTER(CrSolveStats)], _I),
    "cr_set_positions": ([_P, _P, _P], _I),
    "cr_apply_operator": ([_P, _P, _P, _I], _I),
    "cr_precondition": ([_P, _P, _P], _I),
    "cr_coarse_info": ([_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                        C.POINTER(C.c_int)], _I),
    "cr_set_coarse": ([_P, C.c_int, C.c_int], _I),
    "cr_objective": ([_P, _P], _I),
    "cr_wave_potential": ([_P, _P, _P, _I], _I),
    "cr_spread": ([_P, _P, _P, _I], _I),
    "cr_apply_M": ([_P, _P, _P, _I], _I),
    "cr_forces": ([_P, _P, _P, _I], _I),
    "cr_energy": ([_P, _P, C.POINTER(C.c_double)], _I),
    "cr_virial": ([_P, _P, C.POINTER(C.c_double)], _I),
    "cr_neighbor_list": ([_P, C.c_double, _P, _P, _P, C.c_int64, C.POINTER(C.c_int64)], _I),
    "cr_profile": ([_P, _I], _I),
    "cr_profile_read": ([_P, _I, C.POINTER(C.c_int), C.POINTER(C.c_double)], _I),
    "cr_counters": ([_P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)], _I),
    "cr_get_geometry_info": ([_P, C.POINTER(CrGeometryInfo)], _I),
    "cr_body_force_torque": ([_P, _P, _P, _P, _P, _P], _I),
    "cr_brownian_step": ([_P, C.POINTER(CrBrownianParams), C.c_int64, _P, _P, _P, _P], _I),
    "cr_mlp_create": ([C.c_uint64, C.POINTER(_P)], _I),
    "cr_mlp_destroy": ([_P], _I),
    "cr_mlp_last_error": ([_P], C.c_char_p),
    "cr_mlp_get_params": ([_P, C.POINTER(C.c_float)], _I),
    "cr_mlp_set_params": ([_P, C.POINTER(C.c_float)], _I),
    "cr_mlp_get_grads": ([_P, C.POINTER(C.c_float)], _I),
    "cr_mlp_forward": ([_P, _I, _P, _P, _P], _I),
    "cr_mlp_accumulate_grad": ([_P, _I, _P, _P, C.POINTER(C.c_double), _P], _I),
    "cr_mlp_adam": ([_P, C.c_double, C.c_double, _P], _I),
    "cr_mlp_counters": ([_P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)], _I),
    "cr_mlp_set_wait": ([_P, C.c_longlong, _I], _I),
    "cr_set_guess_directions": ([_P, _I, _P], _I),
    "cr_bead_neighbors": ([_P, _P, _P], _I),
    "cr_body_neighbors": ([_P, _P, _P], _I),
    "cr_guess_features": ([_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P], _I),
    "cr_feature_stats": ([_P, _I, _P, _P], _I),
    "cr_feature_pack": ([_P, _I, _P, _P, _P, _P], _I),
    "cr_guess_target": ([_P, _P, _P, C.c_double, _P], _I),
    "cr_neutral_direction": ([_P, _P, _I, C.c_double, _P], _I),
    "cr_batch_compute": ([_I, _P, _P, _P, _P, _P, _P, C.POINTER(CrSolveStats), C.POINTER(C.c_int), _I], _I),
    "cr_batch_create": ([_I, _P, C.POINTER(_P)], _I),
    "cr_batch_destroy": ([_P], _I),
    "cr_batch_last_error": ([_P], C.c_char_p),
    "cr_batch_solve": ([_P, _P, _P, _P, _P, _P, C.POINTER(CrSolveStats), C.POINTER(C.c_int), _I], _I),
    "cr_batch_counters": ([_P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)], _I),
    "cr_batch_phase_ms": ([_P, _D, _D, _D], _I),
    "cr_spread_noalloc": ([C.POINTER(CrDerived), C.c_double, _D, _I, _P, _P, _P, _P], _I),
    "cr_noalloc_last_error": ([], C.c_char_p),
    "cr_util_icosphere_count": ([_I], _I),
    "cr_util_icosphere": ([_I, _D], _I),
    "cr_util_place_spheres": ([_I, _D, _D, C.c_uint64, C.c_int64, _D], _I),
    "cr_util_uniform": ([C.c_uint64, C.c_int64, _D], _I),
}


def lib():
    """Load the library once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH.name} is missing: build it with `python -m conductorrigid_b200.build`"
            )
        L = C.CDLL(str(LIB_PATH))
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def status_string(status: int) -> str:
    try:
        return lib().cr_status_string(status).decode()
    except Exception:  # library not loadable
        return "status"


def check(status: int, where: str, handle=None, allow=(CR_OK,)) -> int:
    if status in allow:
        return status
    msg = ""
    if handle is not None:
        msg = (lib().cr_last_error(handle) or b"").decode()
    raise CrError(status, where, msg)


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def make_params(
    xi: float = 0.5,
    errortol: float = 1e-3,
    field=(0.0, 0.0, 0.0),
    grid=None,
    support: int = 0,
    rcut: float = 0.0,
    gmres_tol: float = 0.0,
    restart: int = 0,
    maxiter: int = 0,
    precision="fp64",
    learned: bool = False,
    precond="diagonal",
) -> CrParams:
    p = CrParams()
    p.field[:] = [float(v) for v in field]
    p.xi = float(xi)
    p.errortol = float(errortol)
    g = [0, 0, 0] if grid is None else ([int(grid)] * 3 if np.isscalar(grid) else [int(v) for v in grid])
    p.grid[:] = g
    p.support = int(support)
    p.rcut = float(rcut)
    p.gmres_tol = float(gmres_tol)
    p.restart = int(restart)
    p.maxiter = int(maxiter)
    p.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    p.learned = int(bool(learned))
    p.precond = PRECONDITIONERS[precond] if isinstance(precond, str) else int(precond)
    return p


def derive_params(params: CrParams, L) -> CrDerived:
    Lv = np.ascontiguousarray(L, dtype=np.float64).reshape(3)
    d = CrDerived()
    check(lib().cr_derive_params(C.byref(params), dptr(Lv), C.byref(d)), "cr_derive_params")
    return d


def build_tables(d: CrDerived, xi: float):
    n = d.n_table + 1
    a = np.zeros(2 * n)
    b = np.zeros(2 * n)
    check(lib().cr_build_tables(C.byref(d), float(xi), dptr(a), dptr(b)), "cr_build_tables")
    return a.reshape(n, 2), b.reshape(n, 2)
