"""Two-level preconditioner (CR_PRECOND_TWO_LEVEL) on the GPU, through the C ABI:
the application against the dense numpy restatement, the coarse level's sizes, and
solves against the oracle with the iteration count against the conductor response."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system():
    from conductorrigid_b200 import systems

    s = systems.spheres(np.ones(40), 1, 0.30, (0.0, 0.0, 1.0), seed=5)
    params = dict(xi=systems.XI_DEFAULT, errortol=1e-5, grid=32, support=9, rcut=4.0)
    return s, params


def _handle(product_lib, s, params, **over):
    from conductorrigid_b200.device import Handle

    kw = dict(params)
    kw.update(over)
    kw.setdefault("field", tuple(s.field))
    h = Handle(product_lib.make_params(**kw), s.L)
    h.set_topology(s.body, s.rigid, s.body_charge)
    h.set_positions(s.pos, s.body_pos)
    return h


def _rel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_two_level_apply_matches_dense(cuda, product_lib, oracle_lib):
    from coarse_ref import TwoLevelRef

    s, params = _system()
    h = _handle(product_lib, s, params, precond="two_level")
    d = h.derived()
    phiq, _ = oracle_lib.tables(oracle_lib.derive(s.L, params["xi"], params["errortol"], params["grid"],
                                                  params["support"], params["rcut"]))
    ref = TwoLevelRef(s, dict(rcut=d.rcut, dr=d.dr, n_table=d.n_table, selfcoeff=d.selfcoeff), phiq, params["xi"])
    info = h.coarse_info()
    assert info["active"] and not info["sparse"] and info["n_coarse"] == 3 * s.n_bodies
    assert info["wave_vectors"] == ref.n_modes
    rng = np.random.default_rng(11)
    for _ in range(2):
        v = rng.standard_normal(s.n_beads + s.n_bodies)
        err = _rel(h.precondition(v), ref.apply(v))
        print(f"\ntwo-level apply: max rel err {err:.2e}")
        assert err < 2e-4  # FP32 pair values, structure factors and C^-1 copy
    h.close()


def test_two_level_inactive_without_rigid_bodies(cuda, product_lib):
    """Free beads only (one-bead bodies, not rigid): no coarse columns, the conductor response."""
    from conductorrigid_b200.systems import ConductorSystem

    s0, params = _system()
    n = 300
    rng = np.random.default_rng(4)
    pos = (rng.random((n, 3)) - 0.5) * s0.L
    s = ConductorSystem(L=s0.L, pos=pos, body=np.arange(n, dtype=np.uint32), rigid=np.zeros(n, dtype=np.uint8),
                        body_charge=np.zeros(n), body_pos=pos.copy(), radius=np.ones(n), field=s0.field)
    h = _handle(product_lib, s, params, precond="two_level")
    assert not h.coarse_info()["active"]
    v = np.random.default_rng(3).standard_normal(s.n_beads + s.n_bodies)
    ref = _handle(product_lib, s, params, precond="conductor")
    assert _rel(h.precondition(v), ref.precondition(v).cpu().numpy()) < 1e-14
    h.close()
    ref.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_two_level_solve_matches_oracle(cuda, product_lib, oracle_lib, precision):
    s, params = _system()
    orc = oracle_lib.Oracle(s, params["xi"], params["errortol"], params["grid"], params["support"], params["rcut"])
    ref = orc.solve(s.field, restart=100, maxiter=4000, tol=1e-11)
    its = {}
    for pc in ("conductor", "two_level"):
        h = _handle(product_lib, s, params, gmres_tol=1e-8, restart=50, maxiter=4000, precision=precision,
                    precond=pc)
        q = h.dev(np.zeros(s.n_beads))
        phi = h.dev(np.zeros(s.n_bodies))
        F, st = h.compute(s.pos, s.body_pos, q, phi)
        h.close()
        eq, ep, ef = _rel(q, ref["q"]), _rel(phi, ref["phi"]), _rel(F, ref["force"])
        print(f"\n{pc} {precision}: iters={st['iterations']} resid={st['final_residual']:.2e} "
              f"err q={eq:.2e} phi={ep:.2e} F={ef:.2e}")
        assert st["converged"] == 1 and st["final_residual"] <= 1e-8
        assert eq < 1e-5 and ep < 1e-5 and ef < 1e-5
        its[pc] = st["iterations"]
    assert 2 * its["two_level"] <= its["conductor"]


def test_two_level_follows_moving_bodies(cuda, product_lib):
    """A new geometry rebuilds the coarse level (captured steps included)."""
    s, params = _system()
    h = _handle(product_lib, s, params, gmres_tol=1e-6, restart=50, maxiter=2000, precision="mixed",
                precond="two_level")
    rng = np.random.default_rng(2)
    for step in range(3):
        q = h.dev(np.zeros(s.n_beads))
        phi = h.dev(np.zeros(s.n_bodies))
        _, st = h.compute(s.pos, s.body_pos, q, phi)
        assert st["converged"] == 1
        shift = 0.02 * rng.standard_normal((s.n_bodies, 3))
        s.pos = s.pos + shift[s.body]
        s.body_pos = s.body_pos + shift
        s.pos -= s.L * np.floor(s.pos / s.L + 0.5)
    assert h.coarse_info()["active"]
    h.close()


def test_sparse_coarse_apply_matches_dense(cuda, product_lib, oracle_lib):
    """The sparse form (near-pair blocks + low-rank wave term, block-Jacobi CG steps)
    against its restatement."""
    from coarse_ref import TwoLevelRef

    s, params = _system()
    h = _handle(product_lib, s, params, precond="two_level")
    h.set_coarse(max_dense=0, pcg_iterations=8)
    d = h.derived()
    phiq, _ = oracle_lib.tables(oracle_lib.derive(s.L, params["xi"], params["errortol"], params["grid"],
                                                  params["support"], params["rcut"]))
    ref = TwoLevelRef(s, dict(rcut=d.rcut, dr=d.dr, n_table=d.n_table, selfcoeff=d.selfcoeff), phiq, params["xi"],
                      pcg_steps=8)
    info = h.coarse_info()
    assert info["active"] and info["sparse"] and info["wave_vectors"] == ref.n_modes
    rng = np.random.default_rng(12)
    for _ in range(2):
        v = rng.standard_normal(s.n_beads + s.n_bodies)
        err = _rel(h.precondition(v), ref.apply(v))
        print(f"\nsparse two-level apply: max rel err {err:.2e}")
        assert err < 2e-4
    h.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_sparse_coarse_solve_matches_oracle(cuda, product_lib, oracle_lib, precision):
    s, params = _system()
    orc = oracle_lib.Oracle(s, params["xi"], params["errortol"], params["grid"], params["support"], params["rcut"])
    ref = orc.solve(s.field, restart=100, maxiter=4000, tol=1e-11)
    its = {}
    for pc, max_dense in (("conductor", 12288), ("two_level", 0)):
        h = _handle(product_lib, s, params, gmres_tol=1e-8, restart=50, maxiter=4000, precision=precision,
                    precond=pc)
        h.set_coarse(max_dense=max_dense, pcg_iterations=8)
        q = h.dev(np.zeros(s.n_beads))
        phi = h.dev(np.zeros(s.n_bodies))
        F, st = h.compute(s.pos, s.body_pos, q, phi)
        h.close()
        eq, ep, ef = _rel(q, ref["q"]), _rel(phi, ref["phi"]), _rel(F, ref["force"])
        print(f"\n{pc} (sparse coarse) {precision}: iters={st['iterations']} resid={st['final_residual']:.2e} "
              f"err q={eq:.2e} phi={ep:.2e} F={ef:.2e}")
        assert st["converged"] == 1 and st["final_residual"] <= 1e-8
        assert eq < 1e-5 and ep < 1e-5 and ef < 1e-5
        its[pc] = st["iterations"]
    assert 3 * its["two_level"] <= 2 * its["conductor"]
