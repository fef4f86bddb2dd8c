"""The virial formulas (tests/virial_ref.py) against finite differences of the oracle's
energy U = 1/2 q.(M q) under stretches of positions and box (CPU)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def case(oracle_lib):
    from oracle import systems as osys

    s, p = osys.workload("plain_small", seed=2, scale=0.3)
    q = np.random.default_rng(5).standard_normal(s.n_beads)
    q -= q.mean()
    return s, p, q


def test_wave_virial_formula_matches_energy_derivative(case, oracle_lib):
    from tests import virial_ref as vr

    s, p, q = case
    orc = oracle_lib.Oracle(s, p["xi"], p["errortol"], p["grid"], p["support"], p["rcut"])
    V, Ek = vr.wave_virial(orc.p, s.pos, s.L, q)
    assert abs(Ek - 0.5 * float(q @ oracle_lib.wave_potential(orc.p, s.pos, q))) < 1e-10 * abs(Ek)
    h = 2e-3
    for a in range(3):
        up = vr.wave_energy_strained(s, p["xi"], p["errortol"], p["grid"], p["support"], p["rcut"], q, a, h)
        dn = vr.wave_energy_strained(s, p["xi"], p["errortol"], p["grid"], p["support"], p["rcut"], q, a, -h)
        fd = -(up - dn) / (2 * h)
        print(f"wave axis {a}: formula {V[a, a]:.6e} finite difference {fd:.6e}")
        assert abs(V[a, a] - fd) < 2e-3 * np.abs(np.diag(V)).max()


def test_real_virial_formula_matches_energy_derivative(case, oracle_lib):
    """The real-space virial against the strain derivative of the real-space energy over a
    fixed pair set.  The reference's truncated kernel is not zero at the cutoff
    (T(rc-) ~ 6e-6 here), so the full energy jumps whenever a pair crosses rc; the virial
    is the derivative of the continuous part, the usual convention for a truncated pair
    sum.  The pair-set energy at zero strain is first pinned to the oracle's."""
    import dataclasses

    from tests import virial_ref as vr

    s, p, q = case
    orc = oracle_lib.Oracle(s, p["xi"], p["errortol"], p["grid"], p["support"], p["rcut"])
    P = orc.p
    i, j = vr.real_pairs(P, s.pos, s.L)
    u0 = vr.real_energy_fixed_pairs(P, s.pos, s.L, q, i, j)
    u_orc = 0.5 * float(q @ (orc.apply_M(q) - oracle_lib.wave_potential(P, s.pos, q))) - 0.5 * P.selfcoeff * float(q @ q)
    assert abs(u0 - u_orc) < 1e-10 * abs(u_orc)
    V = vr.real_virial(P, s.pos, s.L, q)
    h = 1e-3
    for a in range(3):
        f = np.ones(3)
        vals = []
        for sgn in (1.0, -1.0):
            f = np.ones(3)
            f[a] += sgn * h
            vals.append(vr.real_energy_fixed_pairs(P, s.pos * f, np.asarray(s.L) * f, q, i, j))
        fd = -(vals[0] - vals[1]) / (2 * h)
        print(f"real axis {a}: formula {V[a, a]:.6e} finite difference {fd:.6e}")
        assert abs(V[a, a] - fd) < 1e-3 * np.abs(np.diag(V)).max()
