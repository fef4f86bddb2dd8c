"""The FP64 oracle against golden fixtures and known-answer physics (CPU only).

The reference ships no tests or golden vectors and cannot be built here, so the
oracle is pinned by (a) an independent NumPy/SciPy restatement of the reference's
algorithm (tests/golden/make_golden.py) and (b) physics known-answer tests: the
operator reproduces the free-space Coulomb interaction of unit shells, the spectral
Ewald wave-space sum equals the classic Ewald k-sum, the total is independent of the
Ewald split, the forces are the derivative of the energy, and solutions satisfy the
per-body charge constraints.
"""
import math
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def golden_system():
    from conductorrigid_b200.systems import ConductorSystem

    g = np.load(GOLD / "small_system.npz")
    s = ConductorSystem(L=g["L"], pos=g["pos"], body=g["body"], rigid=g["rigid"], body_charge=g["Q"],
                        body_pos=g["body_pos"], radius=np.ones(len(g["Q"])), field=g["E0"])
    return g, s


@pytest.fixture(scope="module")
def gold(oracle_lib, product_lib):
    g, s = golden_system()
    orc = oracle_lib.Oracle(s, float(g["xi"]), float(g["errortol"]), int(g["grid"]), int(g["support"]),
                            float(g["rcut"]))
    return g, s, orc


def test_golden_stages(gold, oracle_lib):
    g, s, orc = gold
    N = s.n_beads
    x = g["x"]
    O = oracle_lib
    assert rel(O.spread(orc.p, g["pos"], x[:N]), g["grid_spread"]) < 1e-13
    assert rel(O.wave_potential(orc.p, g["pos"], x[:N]), g["phi_wave"]) < 1e-13
    assert rel(orc.apply_M(x[:N]), g["Mq"]) < 1e-13
    assert rel(orc.matvec(x), g["y"]) < 1e-13
    assert rel(orc.objective(g["E0"]), g["rhs"]) < 1e-14
    assert rel(orc.precondition(x), g["Px"]) == 0.0
    assert rel(orc.forces(x[:N], g["E0"]), g["force"]) < 1e-13
    t1, t2 = O.tables(orc.p)
    assert rel(t1[:-1], g["table_phiq"]) < 1e-9
    assert rel(t2[:-1], g["table_grad"]) < 1e-8


def test_golden_derivation(oracle_lib):
    rows = np.load(GOLD / "derive_cases.npy")
    for r in rows:
        L, xi, tol = r[0:3], r[3], r[4]
        p = oracle_lib.derive(L, xi, tol)
        assert list(p.N) == [int(v) for v in r[5:8]]
        assert p.P == int(r[8]) and p.P_unclamped == int(r[9])
        np.testing.assert_allclose(list(p.eta), r[10:13], rtol=1e-14)
        assert p.rc == pytest.approx(r[13], rel=1e-15)
        assert p.N_table == int(r[14])
        assert p.prefac == pytest.approx(r[15], rel=1e-13)
        assert p.selfcoeff == pytest.approx(r[16], rel=1e-14)


def test_fft_matches_numpy(oracle_lib):
    rng = np.random.default_rng(3)
    for shape in [(8, 12, 10), (5, 7, 9), (16, 16, 16), (3, 30, 4)]:
        re, im = rng.standard_normal(shape), rng.standard_normal(shape)
        a = re + 1j * im
        fr, fi = oracle_lib.fft3d(re, im, -1)
        assert rel(fr + 1j * fi, np.fft.fftn(a)) < 1e-13
        br, bi = oracle_lib.fft3d(re, im, +1)
        assert rel(br + 1j * bi, np.fft.ifftn(a) * a.size) < 1e-13


def test_neighbor_list_bruteforce(oracle_lib, product_lib):
    from conductorrigid_b200 import systems

    w = systems.workload("plain_small", scale=0.3)
    s = w.system
    count, head, lst = oracle_lib.neighbor_list(s.pos, s.L, 4.0)
    d = s.pos[:, None, :] - s.pos[None, :, :]
    d -= s.L * np.rint(d * (1.0 / s.L))
    d2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
    np.fill_diagonal(d2, np.inf)
    for i in range(s.n_beads):
        ref = np.nonzero(d2[i] < 16.0)[0]
        got = lst[head[i]:head[i] + count[i]]
        assert np.array_equal(ref, got)


def _single_body(L, grid, P, offset=0.013, level=1):
    from conductorrigid_b200 import systems

    v = systems.icosphere(level)
    n = len(v)
    s = systems.ConductorSystem(L=np.array([L] * 3), pos=np.ascontiguousarray(v + offset),
                                body=np.zeros(n, np.uint32), rigid=np.ones(1, np.uint8), body_charge=np.zeros(1),
                                body_pos=np.array([[offset] * 3]), radius=np.ones(1), field=np.array([0, 0, 1.0]))
    return s, v


def _free_space_kernel(v):
    D = np.linalg.norm(v[:, None, :] - v[None, :, :], axis=-1)
    K = np.where(D < 2, (4 - D) / (16 * np.pi), 1 / (4 * np.pi * np.maximum(D, 1e-300)))
    np.fill_diagonal(K, 1 / (4 * np.pi))
    return K


@pytest.mark.parametrize("L,grid,tol", [(24.0, 96, 3e-5), (48.0, 192, 2e-6)])
def test_operator_is_free_space_shell_coulomb(oracle_lib, product_lib, L, grid, tol):
    """k-space + real-space + self reproduce the mutual potential of unit shells
    ((4-d)/(16 pi) overlapping, 1/(4 pi d) apart, 1/(4 pi) self) up to the tin-foil
    periodic term -p.x/(3V) of a neutral charge distribution with dipole p."""
    from conductorrigid_b200 import systems

    s, v = _single_body(L, grid, 11)
    orc = oracle_lib.Oracle(s, systems.XI_DEFAULT, 1e-5, grid, 11, 4.0)
    q = np.random.default_rng(1).standard_normal(len(v))
    q -= q.mean()
    p = (q[:, None] * v).sum(0)
    ref = _free_space_kernel(v) @ q - (v @ p) / (3 * L ** 3)
    assert rel(orc.apply_M(q), ref) < tol


def test_wave_space_equals_classic_ewald(oracle_lib):
    """Spread/FFT/scale/IFFT/contract equals (1/V) sum_{k!=0} j0(k)^2 e^{-k^2/4xi^2}/k^2
    sum_j q_j cos(k.(x_i - x_j)) over the mesh's wave vectors."""
    rng = np.random.default_rng(5)
    L = np.array([8.0, 8.0, 8.0])
    n = 20
    pos = rng.uniform(-4, 4, (n, 3))
    q = rng.standard_normal(n)
    xi = 0.85
    p = oracle_lib.derive(L, xi, 1e-8, grid=32, support=12, rcut=3.0)
    phi = oracle_lib.wave_potential(p, pos, q)
    ks = [np.where(np.arange(32) < 16, np.arange(32), np.arange(32) - 32) * 2 * np.pi / L[d] for d in range(3)]
    kx, ky, kz = np.meshgrid(*ks, indexing="ij")
    k = np.stack([kx.ravel(), ky.ravel(), kz.ravel()], 1)[1:]
    k2 = (k * k).sum(1)
    kk = np.sqrt(k2)
    w = (np.sin(kk) / kk) ** 2 * np.exp(-k2 / (4 * xi * xi)) / k2
    phase = k @ pos.T
    rho_c = (np.cos(phase) * q).sum(1)
    rho_s = (np.sin(phase) * q).sum(1)
    ref = (w[:, None] * (np.cos(phase) * rho_c[:, None] + np.sin(phase) * rho_s[:, None])).sum(0) / np.prod(L)
    assert rel(phi, ref) < 1e-6


def test_ewald_split_independence(oracle_lib, product_lib):
    """M q is the same physical operator for different splitting parameters (for a
    neutral charge vector; a net charge adds the split-dependent background shift)."""
    from conductorrigid_b200 import systems

    w = systems.workload("plain_small", scale=0.3)
    s = w.system
    q = np.random.default_rng(2).standard_normal(s.n_beads)
    q -= q.mean()
    out = []
    for xi in (1.0, 1.3):
        orc = oracle_lib.Oracle(s, xi, 1e-11, 96)
        out.append(orc.apply_M(q))
    assert rel(out[0], out[1]) < 1e-5


def test_forces_are_energy_gradient(oracle_lib, product_lib):
    """F_i = -dU/dx_i at fixed charges, U = q.Mq/2 - sum q_i E0.x_i (central differences)."""
    from conductorrigid_b200 import systems

    w = systems.workload("plain_small", scale=0.2)
    s = w.system
    p = w.params
    orc = oracle_lib.Oracle(s, p["xi"], p["errortol"], p["grid"], p["support"], p["rcut"])
    rng = np.random.default_rng(4)
    q = rng.standard_normal(s.n_beads)
    E0 = np.array([0.3, -0.4, 1.0])
    F = orc.forces(q, E0)
    h = orc.p.h[0]

    def energy(pos):
        orc.set_positions(pos, s.body_pos)
        return 0.5 * q @ orc.apply_M(q) - q @ (pos @ E0)

    delta = 1e-5
    checked = 0
    for i in rng.permutation(s.n_beads):
        u = (s.pos[i] + 0.5 * s.L) / s.L * orc.p.N[0]
        if np.any(np.abs((u - np.trunc(u)) - 0.5) < 1e-3):  # window switch nearby
            continue
        for d in range(3):
            pp, pm = s.pos.copy(), s.pos.copy()
            pp[i, d] += delta
            pm[i, d] -= delta
            fd = -(energy(pp) - energy(pm)) / (2 * delta)
            assert fd == pytest.approx(F[i, d], rel=2e-4, abs=2e-5 * np.abs(F).max())
        checked += 1
        if checked == 4:
            break
    orc.set_positions(s.pos, s.body_pos)
    assert checked == 4 and h > 0


def test_solution_constraints(oracle_lib, product_lib):
    from conductorrigid_b200 import systems

    w = systems.workload("polydisperse_204k", scale=0.004)
    s = w.system
    p = w.params
    orc = oracle_lib.Oracle(s, p["xi"], p["errortol"], 48, p["support"], p["rcut"])
    r = orc.solve(s.field, restart=60, maxiter=3000, tol=1e-10)
    assert r["true_rel"] < 1e-9
    sums = np.bincount(s.body, weights=r["q"], minlength=s.n_bodies)
    np.testing.assert_allclose(sums, s.body_charge, atol=1e-9)
    # equipotential: M q - (r - R).E0 equals the body potential on every bead
    Mq = orc.apply_M(r["q"])
    rr = s.pos - s.body_pos[s.body]
    rr -= s.L * np.rint(rr / s.L)
    pot = Mq - rr @ s.field
    np.testing.assert_allclose(pot, r["phi"][s.body], atol=1e-8 * np.abs(pot).max())
    # net force balance: internal forces cancel up to the mesh discretisation
    F = r["force"]
    assert np.abs(F.sum(0) - s.body_charge.sum() * s.field).max() < 1e-4 * np.abs(F).sum(0).max()


def test_linear_response(oracle_lib, product_lib):
    """Charges induced on neutral conductors scale linearly with the field."""
    from conductorrigid_b200 import systems

    w = systems.workload("plain_small", scale=0.2)
    s = w.system
    p = w.params
    orc = oracle_lib.Oracle(s, p["xi"], p["errortol"], 32, p["support"], p["rcut"])
    r1 = orc.solve(np.array([0.0, 0.0, 1.0]), restart=60, maxiter=3000, tol=1e-11)
    r2 = orc.solve(np.array([0.0, 0.0, 2.5]), restart=60, maxiter=3000, tol=1e-11)
    assert rel(r2["q"], 2.5 * r1["q"]) < 1e-8
