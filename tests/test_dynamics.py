"""Rigid-body Brownian stepper: the NumPy restatement on CPU, the CUDA kernels against it on GPU."""
import numpy as np
import pytest

import brownian_ref as br


def _system(scale=0.3):
    from conductorrigid_b200 import systems

    return systems.workload("plain_small", scale=scale).system


def _mimg(d, L):
    L = np.asarray(L)
    return d - L * np.rint(d / L)


def test_counter_normals_statistics():
    g = np.array([br.normals6(7, s, b) for s in range(40) for b in range(100)]).ravel()
    assert abs(g.mean()) < 0.03 and abs(g.std() - 1.0) < 0.03
    # a pure function of (seed, step, body)
    assert np.array_equal(br.normals6(7, 3, 11), br.normals6(7, 3, 11))
    assert not np.array_equal(br.normals6(7, 3, 11), br.normals6(7, 4, 11))
    assert not np.array_equal(br.normals6(7, 3, 11), br.normals6(8, 3, 11))


def test_repulsion_is_pairwise_and_opens_gaps():
    s = _system()
    B = s.n_bodies
    Fr = br.repulsion(s.body_pos, np.ones(B), s.L, 100.0, 0.3)
    assert np.abs(Fr.sum(0)).max() < 1e-9  # equal and opposite
    bpos = s.body_pos.copy()
    pos = s.pos.copy()
    for step in range(200):
        pos, bpos, _ = br.brownian_step(pos, s.body, s.rigid, bpos, np.ones(B), np.zeros_like(pos), s.L, step, kT=0.0,
                                        dt=0.05, k_rep=100.0, gap=0.3)
    D = _mimg(bpos[None] - bpos[:, None], s.L)
    d = np.linalg.norm(D, axis=-1) + np.eye(B) * 1e9
    d0 = np.linalg.norm(_mimg(s.body_pos[None] - s.body_pos[:, None], s.L), axis=-1) + np.eye(B) * 1e9
    assert d.min() > d0.min()


def test_restatement_keeps_bodies_rigid_and_drifts_with_force():
    s = _system()
    B = s.n_bodies
    F = np.zeros((s.n_beads, 3))
    F[:, 2] = 1.0  # uniform force: no torque about the centre of a symmetric shell
    pos, bpos, moves = br.brownian_step(s.pos, s.body, s.rigid, s.body_pos, np.ones(B), F, s.L, step=0, kT=0.0)
    n_b = np.bincount(s.body, minlength=B)
    dz = _mimg(bpos - s.body_pos, s.L)
    assert np.allclose(dz[:, 2], n_b / (6 * np.pi) * 1e-3, rtol=1e-12, atol=1e-15)
    assert np.allclose(dz[:, :2], 0.0, atol=1e-15)
    # thermal step: bead-centre distances preserved
    pos, bpos, moves = br.brownian_step(s.pos, s.body, s.rigid, s.body_pos, np.ones(B), 0 * F, s.L, step=1)
    d0 = np.linalg.norm(_mimg(s.pos - s.body_pos[s.body], s.L), axis=1)
    d1 = np.linalg.norm(_mimg(pos - bpos[s.body], s.L), axis=1)
    assert np.abs(d1 - d0).max() < 1e-13
    assert (np.abs(pos) <= 0.5 * np.asarray(s.L)).all()
    assert moves[:, 1].mean() > 0


@pytest.mark.gpu
def test_body_force_torque_matches_restatement(cuda, product_lib):
    from conductorrigid_b200 import _lib
    from conductorrigid_b200.device import Handle

    s = _system()
    h = Handle(_lib.make_params(field=(0, 0, 1), xi=0.85, errortol=1e-5, grid=(32, 32, 32), support=9, rcut=4.0),
               s.L)
    h.set_topology(s.body, s.rigid, s.body_charge)
    F = np.random.default_rng(3).standard_normal((s.n_beads, 3))
    bf, bt = h.body_force_torque(s.pos, s.body_pos, F)
    rf, rt = br.body_force_torque(s.pos, s.body, s.body_pos, F, s.L)
    assert np.abs(bf.cpu().numpy() - rf).max() < 1e-12
    assert np.abs(bt.cpu().numpy() - rt).max() < 1e-12
    h.close()


@pytest.mark.gpu
def test_brownian_steps_match_restatement(cuda, product_lib):
    from conductorrigid_b200 import _lib
    from conductorrigid_b200.device import Handle

    torch = cuda
    s = _system()
    h = Handle(_lib.make_params(field=(0, 0, 1), xi=0.85, errortol=1e-5, grid=(32, 32, 32), support=9, rcut=4.0),
               s.L)
    h.set_topology(s.body, s.rigid, s.body_charge)
    rng = np.random.default_rng(5)
    radius = 1.0 + 0.1 * rng.random(s.n_bodies)
    F = 20.0 * rng.standard_normal((s.n_beads, 3))
    pos = torch.tensor(s.pos, device="cuda", dtype=torch.float64).contiguous()
    bpos = torch.tensor(s.body_pos, device="cuda", dtype=torch.float64).contiguous()
    rp, rb = s.pos.copy(), s.body_pos.copy()
    for step in range(4):
        kr = 300.0 if step % 2 else 0.0  # steric repulsion on every other step
        h.brownian_step(step, radius, F, pos, bpos, dt=2e-3, kT=1.5, viscosity=0.8, seed=11, repulsion=kr,
                        contact_gap=0.5)
        rp, rb, _ = br.brownian_step(rp, s.body, s.rigid, rb, radius, F, s.L, step, dt=2e-3, kT=1.5, viscosity=0.8,
                                     seed=11, k_rep=kr, gap=0.5)
    assert np.abs(_mimg(pos.cpu().numpy() - rp, s.L)).max() < 1e-11
    assert np.abs(_mimg(bpos.cpu().numpy() - rb, s.L)).max() < 1e-11
    # moved noticeably, stayed rigid
    assert np.abs(_mimg(rb - s.body_pos, s.L)).max() > 1e-2
    h.close()
