"""Box change (parameters re-derived for a new box on a live handle) and the
electrostatic energy 1/2 q.(M q) against the FP64 oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system():
    from conductorrigid_b200 import systems

    return systems.workload("plain_small", scale=0.3).system


def _moved_box(s, f):
    """The same rigid bodies in a box scaled by f: centres scaled, bead offsets kept."""
    L2 = np.asarray(s.L) * f
    off = s.pos - s.body_pos[s.body]
    off -= np.asarray(s.L) * np.rint(off / np.asarray(s.L))
    c2 = s.body_pos * f
    p2 = c2[s.body] + off
    p2 -= L2 * np.floor((p2 + 0.5 * L2) / L2)
    return L2, p2, c2


def test_box_change_matches_fresh_handle(cuda, product_lib):
    from conductorrigid_b200 import _lib
    from conductorrigid_b200.device import Handle

    s = _system()
    P = _lib.make_params(field=tuple(s.field), xi=0.85, errortol=1e-5, rcut=4.0, gmres_tol=1e-10, restart=100,
                         maxiter=4000, precision="fp64", precond="conductor")
    h = Handle(P, s.L)
    h.set_topology(s.body, s.rigid, s.body_charge)
    q = h.dev(np.zeros(s.n_beads))
    phi = h.dev(np.zeros(s.n_bodies))
    h.compute(s.pos, s.body_pos, q, phi)
    g1 = tuple(h.derived().grid)
    L2, p2, c2 = _moved_box(s, 1.3)
    h.set_params(P, L2)
    g2 = tuple(h.derived().grid)
    assert g2 != g1  # mesh re-derived for the larger box
    q.zero_()
    phi.zero_()
    F, st = h.compute(p2, c2, q, phi)
    assert st["converged"] == 1
    f = Handle(P, L2)
    f.set_topology(s.body, s.rigid, s.body_charge)
    qf = f.dev(np.zeros(s.n_beads))
    pf = f.dev(np.zeros(s.n_bodies))
    Ff, _ = f.compute(p2, c2, qf, pf)
    for a, b in ((q, qf), (phi, pf), (F, Ff)):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max()
    h.close()
    f.close()


def test_box_change_matches_oracle(cuda, product_lib, oracle_lib):
    """After cr_set_params with a new box, the live handle's operator, forces and solution
    are the oracle's at that box (parameters re-derived by the oracle from the same inputs,
    ConductorRigid.cc:116-379)."""
    import dataclasses

    from conductorrigid_b200 import _lib
    from conductorrigid_b200.device import Handle

    s = _system()
    P = _lib.make_params(field=tuple(s.field), xi=0.85, errortol=1e-5, rcut=4.0, gmres_tol=1e-10, restart=100,
                         maxiter=4000, precision="fp64", precond="conductor")
    h = Handle(P, s.L)
    h.set_topology(s.body, s.rigid, s.body_charge)
    q = h.dev(np.zeros(s.n_beads))
    phi = h.dev(np.zeros(s.n_bodies))
    h.compute(s.pos, s.body_pos, q, phi)
    L2, p2, c2 = _moved_box(s, 1.3)
    h.set_params(P, L2)
    s2 = dataclasses.replace(s, L=L2, pos=p2, body_pos=c2)
    orc = oracle_lib.Oracle(s2, 0.85, 1e-5, None, 0, 4.0)
    d = h.derived()
    assert list(d.grid) == list(orc.p.N) and d.support == orc.p.P
    q.zero_()
    phi.zero_()
    F, st = h.compute(p2, c2, q, phi)
    assert st["converged"] == 1
    x = np.random.default_rng(8).standard_normal(s.n_beads + s.n_bodies)
    y = orc.matvec(x)
    assert np.abs(h.apply_operator(x).cpu().numpy() - y).max() <= 1e-11 * np.abs(y).max()
    ref = orc.solve_tight(s2.field, tol=1e-12)
    for a, b in ((q, ref["q"]), (phi, ref["phi"]), (F, ref["force"])):
        a = a.cpu().numpy()
        assert np.abs(a - b).max() <= 1e-7 * np.abs(b).max()
    h.close()


def test_energy_matches_oracle(cuda, product_lib, oracle_lib):
    from conductorrigid_b200 import _lib
    from conductorrigid_b200.device import Handle

    s = _system()
    orc = oracle_lib.Oracle(s, 0.85, 1e-5, 48, 9, 4.0)
    h = Handle(_lib.make_params(field=tuple(s.field), xi=0.85, errortol=1e-5, grid=48, support=9, rcut=4.0), s.L)
    h.set_topology(s.body, s.rigid, s.body_charge)
    h.set_positions(s.pos, s.body_pos)
    q = np.random.default_rng(4).standard_normal(s.n_beads)
    U = h.energy(q)
    U_ref = 0.5 * float(q @ orc.apply_M(q))
    assert abs(U - U_ref) <= 1e-10 * abs(U_ref)
    assert U > 0  # the shell interaction is positive definite
    h.close()
