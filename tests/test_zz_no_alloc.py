"""cr_spread_noalloc: charge spreading for callers that cannot allocate device memory.

Such callers (an engine that owns every device allocation through its own pool, or a
time-step loop where cudaMalloc/cudaFree would synchronise the device) get a spread
whose scratch sits in a fixed file-scope device array.  These tests call it through the
C ABI and check it against cr_spread, the existing entry point, within the FP64 operator
tolerance used by the other parity tests, on two calls in a row (the array keeps the
previous call's contents, so the second call also checks that each call clears it).
The shapes cover a mesh that is a multiple of the 8-node tile (64^3), one that is not
(60^3, partial edge tiles), one smaller than a tile's halo (12^3: the halo wraps onto
the mesh several times), odd and even supports up to the maximum of 16, and positions
shifted by whole box lengths.  This file is collected last so that a failure here comes
after every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _handle(product_lib, s, p, grid, support):
    from conductorrigid_b200.device import Handle

    params = product_lib.make_params(xi=p["xi"], errortol=p["errortol"], grid=grid, support=support, rcut=p["rcut"])
    h = Handle(params, s.L)
    h.set_topology(s.body, s.rigid, s.body_charge)
    h.set_positions(s.pos, s.body_pos)
    return h


def _noalloc(product_lib, h, s, xi, pos_t, q_t, grid_t, n=None):
    d = h.derived()
    L = np.ascontiguousarray(s.L, dtype=np.float64)
    return product_lib.lib().cr_spread_noalloc(C.byref(d), float(xi), product_lib.dptr(L),
                                               int(s.n_beads if n is None else n), C.c_void_p(pos_t.data_ptr()),
                                               C.c_void_p(q_t.data_ptr()), C.c_void_p(grid_t.data_ptr()), None)


@pytest.fixture(scope="module")
def system(cuda, product_lib):
    from conductorrigid_b200 import systems

    w = systems.workload("plain_small")
    return w.system, w.params


@pytest.mark.parametrize("grid,support,shift", [(64, 9, 0), (60, 8, 0), (60, 11, 1), (64, 16, -1), (12, 11, 2)])
def test_spread_noalloc_matches_cr_spread_twice(system, product_lib, cuda, grid, support, shift):
    s, p = system
    torch = cuda
    h = _handle(product_lib, s, p, grid, support)
    d = h.derived()
    assert d.support == support and d.grid[0] == grid
    # the same beads, moved by whole box lengths (the entry point wraps them itself)
    pos_t = h.dev(s.pos + shift * s.L).reshape(-1, 3)
    grid_t = torch.empty(d.grid[0] * d.grid[1] * d.grid[2], dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(21 + grid + support)
    for call in range(2):
        q = rng.standard_normal(s.n_beads)
        q_t = h.dev(q)
        st = _noalloc(product_lib, h, s, p["xi"], pos_t, q_t, grid_t)
        assert st == product_lib.CR_OK, product_lib.lib().cr_noalloc_last_error()
        ref = h.spread(q).cpu().numpy().ravel()
        assert _rel(grid_t.cpu().numpy(), ref) < 1e-12, f"call {call}"
    h.close()


def test_spread_noalloc_rejects_non_finite_position(system, product_lib, cuda):
    s, p = system
    torch = cuda
    h = _handle(product_lib, s, p, 64, 9)
    d = h.derived()
    bad = s.pos.copy()
    bad[123, 2] = np.nan
    pos_t = h.dev(bad).reshape(-1, 3)
    q_t = h.dev(np.ones(s.n_beads))
    grid_t = torch.empty(d.grid[0] * d.grid[1] * d.grid[2], dtype=torch.float64, device="cuda")
    assert _noalloc(product_lib, h, s, p["xi"], pos_t, q_t, grid_t) == product_lib.CR_NUMERICAL
    assert b"non-finite" in product_lib.lib().cr_noalloc_last_error()
    # the next call with valid positions is unaffected
    pos_t = h.dev(s.pos).reshape(-1, 3)
    assert _noalloc(product_lib, h, s, p["xi"], pos_t, q_t, grid_t) == product_lib.CR_OK
    assert _rel(grid_t.cpu().numpy(), h.spread(np.ones(s.n_beads)).cpu().numpy().ravel()) < 1e-12
    h.close()


def test_spread_noalloc_rejects_oversize(system, product_lib, cuda):
    s, p = system
    h = _handle(product_lib, s, p, 64, 9)
    d = h.derived()
    L = np.ascontiguousarray(s.L, dtype=np.float64)
    big = 262144 + 1
    st = product_lib.lib().cr_spread_noalloc(C.byref(d), float(p["xi"]), product_lib.dptr(L), big,
                                             C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), None)
    assert st == product_lib.CR_BAD_PARAM
    assert b"CR_NOALLOC_MAX_BEADS" in product_lib.lib().cr_noalloc_last_error()
    h.close()
