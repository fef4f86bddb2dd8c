"""Mesh tiling: every tile edge and spread mode gives the default operator (FP64, up to
the summation order of the spreading atomics), an oversize tile is refused, and the
autotuner's choice solves to the same result."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(grid, support):
    from conductorrigid_b200 import _lib, systems
    from conductorrigid_b200.device import Handle

    s = systems.workload("plain_small", scale=0.3).system
    P = _lib.make_params(field=tuple(s.field), xi=0.85, errortol=1e-5, grid=grid, support=support, rcut=4.0,
                         gmres_tol=1e-8, restart=50, maxiter=4000, precision="mixed", precond="conductor")
    h = Handle(P, s.L)
    h.set_topology(s.body, s.rigid, s.body_charge)
    return s, h


@pytest.mark.parametrize("grid,support", [(50, 9), (48, 11), (45, 7)])
def test_every_tiling_gives_the_default_operator(cuda, product_lib, grid, support):
    from conductorrigid_b200 import _lib

    s, h = _setup(grid, support)
    x = np.random.default_rng(1).standard_normal(s.n_beads + s.n_bodies)
    h.set_positions(s.pos, s.body_pos)
    ref = h.apply_operator(x, _lib.CR_FP64).cpu().numpy()
    ref32 = h.apply_operator(x, _lib.CR_FP32).cpu().numpy()
    for tile, mode in ((8, 1), (4, 1), (6, 1), (12, 1), (16, 1)):
        h.set_tiling(tile, mode)
        h.set_positions(s.pos, s.body_pos)
        assert h.geometry_info()["tile_edge"] == tile
        y = h.apply_operator(x, _lib.CR_FP64).cpu().numpy()
        assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max(), (tile, mode)
        y32 = h.apply_operator(x, _lib.CR_FP32).cpu().numpy()
        assert np.abs(y32 - ref32).max() <= 1e-5 * np.abs(ref32).max(), (tile, mode)
    with pytest.raises(_lib.CrError):
        h.set_tiling(32, 1)  # (32 + P - 1)^3 FP64 halo exceeds shared memory
    h.set_positions(s.pos, s.body_pos)
    y = h.apply_operator(x, _lib.CR_FP64).cpu().numpy()  # still usable at the previous tiling
    assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()
    h.close()


def test_autotuned_solve_matches_default(cuda, product_lib):
    s, h = _setup(50, 9)
    q0 = h.dev(np.zeros(s.n_beads))
    p0 = h.dev(np.zeros(s.n_bodies))
    F0, _ = h.compute(s.pos, s.body_pos, q0, p0)
    choice = h.autotune(s.pos, s.body_pos, reps=3)
    assert choice["tile_edge"] in (4, 6, 8, 12, 16) and choice["mesh_ms"] > 0
    q1 = h.dev(np.zeros(s.n_beads))
    p1 = h.dev(np.zeros(s.n_bodies))
    F1, st = h.compute(s.pos, s.body_pos, q1, p1)
    assert st["converged"] == 1
    for a, b in ((q0, q1), (p0, p1), (F0, F1)):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.abs(a - b).max() <= 1e-6 * np.abs(a).max()
    h.close()
