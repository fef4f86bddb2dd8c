"""cr_spread_noalloc: charge spreading for callers that cannot allocate device memory.

Such callers (an engine that owns every device allocation through its own pool, or a
time-step loop where cudaMalloc/cudaFree would synchronise the device) get a spread
whose scratch sits in a fixed file-scope device array.  These tests call it through the
C ABI and check it against cr_spread, the existing entry point, within the FP64 operator
tolerance used by the other parity tests, on two calls in a row (the array keeps the
previous call's contents, so the second call also checks that each call clears it).
This file is collected last so that a failure here comes after every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def setup(cuda, product_lib):
    from conductorrigid_b200 import systems
    from conductorrigid_b200.device import Handle

    w = systems.workload("plain_small")
    s, p = w.system, w.params
    params = product_lib.make_params(**{k: p[k] for k in ("xi", "errortol", "grid", "support", "rcut")})
    h = Handle(params, s.L)
    h.set_topology(s.body, s.rigid, s.body_charge)
    h.set_positions(s.pos, s.body_pos)
    yield s, p, h
    h.close()


def _noalloc(product_lib, h, s, xi, pos_t, q_t, grid_t):
    d = h.derived()
    L = np.ascontiguousarray(s.L, dtype=np.float64)
    st = product_lib.lib().cr_spread_noalloc(C.byref(d), float(xi), product_lib.dptr(L), int(s.n_beads),
                                             C.c_void_p(pos_t.data_ptr()), C.c_void_p(q_t.data_ptr()),
                                             C.c_void_p(grid_t.data_ptr()), None)
    return st


def test_spread_noalloc_matches_cr_spread_twice(setup, product_lib, cuda):
    s, p, h = setup
    torch = cuda
    d = h.derived()
    pos_t = h.dev(s.pos).reshape(-1, 3)
    grid_t = torch.empty(d.grid[0] * d.grid[1] * d.grid[2], dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(21)
    for call in range(2):
        q = rng.standard_normal(s.n_beads)
        q_t = h.dev(q)
        st = _noalloc(product_lib, h, s, p["xi"], pos_t, q_t, grid_t)
        assert st == product_lib.CR_OK, product_lib.lib().cr_noalloc_last_error()
        ref = h.spread(q).cpu().numpy().ravel()
        assert _rel(grid_t.cpu().numpy(), ref) < 1e-12, f"call {call}"


def test_spread_noalloc_rejects_oversize(setup, product_lib, cuda):
    s, p, h = setup
    d = h.derived()
    L = np.ascontiguousarray(s.L, dtype=np.float64)
    big = 262144 + 1
    st = product_lib.lib().cr_spread_noalloc(C.byref(d), float(p["xi"]), product_lib.dptr(L), big,
                                             C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), None)
    assert st == product_lib.CR_BAD_PARAM
    assert b"CR_NOALLOC_MAX_BEADS" in product_lib.lib().cr_noalloc_last_error()
