"""Learned initial guess on the GPU: neighbour searches, features and transport term
against a NumPy restatement, guess directions leave the fixed point unchanged, and the
trained guess lowers the GMRES iteration count of time stepping against the plain
warm-started solver on the same trajectory."""
import numpy as np
import pytest

import brownian_ref as br
import guess_ref as gr

pytestmark = pytest.mark.gpu


def _system(n_bodies=120, seed=3):
    from conductorrigid_b200 import systems

    return systems.spheres(np.ones(n_bodies), 1, 0.35, (0.0, 0.0, 1.0), seed=seed)


def _params(s, **kw):
    from conductorrigid_b200 import _lib, systems

    grid = systems.smooth_at_least(int(np.ceil(5.2 * s.L[0])))
    base = dict(field=tuple(s.field), xi=systems.XI_DEFAULT, errortol=1e-5, grid=(grid,) * 3, support=9, rcut=4.0,
                gmres_tol=1e-6, restart=50, maxiter=4000, precision="mixed", precond="conductor")
    base.update(kw)
    return _lib.make_params(**base)


def _moved(s, seed=9):
    rng = np.random.default_rng(seed)
    F = rng.standard_normal((s.n_beads, 3))
    pos, bpos, _ = br.brownian_step(s.pos, s.body, s.rigid, s.body_pos, np.ones(s.n_bodies), F, s.L, step=0,
                                    seed=seed)
    return pos, bpos


def test_neighbor_searches_pick_the_nearest(cuda, product_lib):
    from conductorrigid_b200 import _lib
    from conductorrigid_b200.device import Handle
    from conductorrigid_b200.dynamics import BEAD_K, BODY_K, _p

    torch = cuda
    s = _system()
    h = Handle(_params(s), s.L)
    h.set_topology(s.body, s.rigid, s.body_charge)
    pos = h.dev(s.pos)
    bpos = h.dev(s.body_pos)
    bn = torch.empty(s.n_beads, BEAD_K, dtype=torch.int32, device="cuda")
    kn = torch.empty(s.n_bodies, BODY_K, dtype=torch.int32, device="cuda")
    assert _lib.lib().cr_bead_neighbors(h.h, _p(pos), _p(bn)) == 0
    assert _lib.lib().cr_body_neighbors(h.h, _p(bpos), _p(kn)) == 0
    bn, kn = bn.cpu().numpy(), kn.cpu().numpy()
    for i in range(0, s.n_beads, 7):
        mates = np.nonzero(s.body == s.body[i])[0]
        mates = mates[mates != i]
        d = np.sort(np.linalg.norm(gr.mimg(s.pos[mates] - s.pos[i], s.L), axis=1))[:BEAD_K]
        got = np.sort(np.linalg.norm(gr.mimg(s.pos[bn[i]] - s.pos[i], s.L), axis=1))
        assert np.allclose(got, d, rtol=0, atol=1e-12)
        assert s.body[bn[i]].tolist() == [s.body[i]] * BEAD_K
    for b in range(s.n_bodies):
        d = np.linalg.norm(gr.mimg(s.body_pos - s.body_pos[b], s.L), axis=1)
        d[b] = np.inf
        got = np.linalg.norm(gr.mimg(s.body_pos[kn[b]] - s.body_pos[b], s.L), axis=1)
        assert np.allclose(got, np.sort(d)[:BODY_K], rtol=0, atol=1e-12)
    h.close()


def test_features_and_transport_match_restatement(cuda, product_lib):
    from conductorrigid_b200 import _lib
    from conductorrigid_b200.device import Handle
    from conductorrigid_b200.dynamics import BEAD_K, BODY_K, _p

    torch = cuda
    s = _system()
    h = Handle(_params(s), s.L)
    h.set_topology(s.body, s.rigid, s.body_charge)
    rng = np.random.default_rng(2)
    q_prev = rng.standard_normal(s.n_beads) * 0.1
    pos, bpos = _moved(s)
    t = {k: h.dev(v) for k, v in dict(q=q_prev, pp=s.pos, bp=s.body_pos, p=pos, b=bpos, r=np.ones(s.n_bodies)).items()}
    bn = torch.empty(s.n_beads, BEAD_K, dtype=torch.int32, device="cuda")
    kn = torch.empty(s.n_bodies, BODY_K, dtype=torch.int32, device="cuda")
    feat = torch.empty(s.n_beads, 48, dtype=torch.float32, device="cuda")
    tr = torch.empty(s.n_beads, dtype=torch.float64, device="cuda")
    L = _lib.lib()
    assert L.cr_bead_neighbors(h.h, _p(t["pp"]), _p(bn)) == 0
    assert L.cr_body_neighbors(h.h, _p(t["b"]), _p(kn)) == 0
    assert L.cr_guess_features(h.h, _p(t["r"]), _p(bn), _p(kn), _p(t["q"]), _p(t["pp"]), _p(t["bp"]), _p(t["p"]),
                               _p(t["b"]), _p(feat), _p(tr)) == 0
    f_ref, s_ref = gr.features(q_prev, s.pos, s.body_pos, pos, bpos, s.body, s.body_charge, np.ones(s.n_bodies),
                               bn.cpu().numpy(), kn.cpu().numpy(), s.field, s.L)
    assert np.abs(tr.cpu().numpy() - s_ref).max() <= 1e-9 * max(np.abs(s_ref).max(), 1e-300)
    f = feat.cpu().numpy()
    scale = np.maximum(np.abs(f_ref).max(0), 1e-30)
    assert (np.abs(f - f_ref).max(0) <= 2e-6 * scale + 1e-30).all()
    # neutral direction: per-body sums vanish, potential rows zero
    d = torch.empty(s.n_beads + s.n_bodies, dtype=torch.float64, device="cuda")
    assert L.cr_neutral_direction(h.h, _p(tr), 0, 2.0, _p(d)) == 0
    d = d.cpu().numpy()
    assert np.abs(np.bincount(s.body, d[:s.n_beads])).max() < 1e-12
    assert not np.any(d[s.n_beads:])
    h.close()


def test_guess_directions_keep_the_solution(cuda, product_lib):
    from conductorrigid_b200.device import Handle

    torch = cuda
    s = _system()
    pos, bpos = _moved(s)
    sols = []
    for learned in (False, True):
        h = Handle(_params(s, learned=learned), s.L)
        h.set_topology(s.body, s.rigid, s.body_charge)
        q = torch.zeros(s.n_beads, dtype=torch.float64, device="cuda")
        phi = torch.zeros(s.n_bodies, dtype=torch.float64, device="cuda")
        h.compute(s.pos, s.body_pos, q, phi)  # previous step
        if learned:
            from conductorrigid_b200.dynamics import LearnedGuess

            g = LearnedGuess(h, np.ones(s.n_bodies), use_network=False)
            assert g.prepare(q.clone(), h.dev(s.pos).reshape(-1, 3), h.dev(s.body_pos).reshape(-1, 3),
                             h.dev(pos).reshape(-1, 3), h.dev(bpos).reshape(-1, 3), phi.clone()) == 2
        F, st = h.compute(pos, bpos, q, phi)
        assert st["converged"] == 1 and st["final_residual"] <= 1e-6
        if learned:
            assert st["learned_residual"] < st["initial_residual"] and st["used_learned_guess"] == 1
        sols.append((q.cpu().numpy(), phi.cpu().numpy(), F.cpu().numpy()))
        h.close()
    for a, b in zip(sols[0], sols[1]):
        assert np.abs(a - b).max() <= 1e-5 * np.abs(a).max()


def test_learned_guess_in_time_stepping(cuda, product_lib):
    """Paired trajectory (phi 0.10): the learned solver's start never exceeds the warm
    start's residual, its solutions match the plain solver's, and the network, trained
    online on the first solves, predicts part of the next solves' charge change.  The
    GMRES iteration counts of both solvers are printed: on these systems the start does
    not change them (the iterations are set by the operator's spectrum)."""
    from conductorrigid_b200.dynamics import paired_run

    s = systems_small(0.10)
    steps, train = 24, 12
    out, guess, _ = paired_run(_params(s), _params(s, learned=True), s, np.ones(s.n_bodies), steps,
                               train_solves=train, seed=7)
    for k, o in enumerate(out):
        print(f"step {k:3d} plain it {o['plain']['iterations']:4d} r0 {o['plain']['initial_residual']:.2e} | "
              f"learned it {o['learned']['iterations']:4d} r0 {o['learned']['initial_residual']:.2e} "
              f"-> {o['learned']['learned_residual']:.2e}")
    print("explained (training)", np.round(guess.explained, 3).tolist())
    print("explained (held out)", np.round(guess.heldout, 3).tolist())
    assert guess.trained == train
    assert all(o["learned"]["converged"] == 1 and o["plain"]["converged"] == 1 for o in out)
    for o in out[1:]:
        assert o["learned"]["learned_residual"] <= min(1.0, o["learned"]["initial_residual"]) * (1 + 1e-9)
    tail = out[train + 1:]
    it_plain = np.mean([o["plain"]["iterations"] for o in tail])
    it_learned = np.mean([o["learned"]["iterations"] for o in tail])
    print(f"iterations after training: plain {it_plain:.1f} learned {it_learned:.1f}")
    assert np.mean(guess.heldout[-(steps - train - 1):]) > 0.0


def systems_small(phi):
    from conductorrigid_b200 import systems

    return systems.spheres(np.ones(150), 1, phi, (0.0, 0.0, 1.0), seed=5)


def test_learned_correction_in_time_stepping(cuda, product_lib):
    """The third arm: learned start plus the learned preconditioner correction, trained
    online.  Every solve converges; a solve that used the correction had passed its
    initial-residual test (one-step reduction below the plain preconditioner's)."""
    from conductorrigid_b200.dynamics import paired_run

    s = systems_small(0.20)
    steps, train = 16, 8
    out, guess, corr = paired_run(_params(s), _params(s, learned=True), s, np.ones(s.n_bodies), steps,
                                  train_solves=train, seed=3, corrected=True)
    assert corr.trained == train and len(corr.losses) == train
    for k, o in enumerate(out):
        c = o["corrected"]
        print(f"step {k:3d} plain it {o['plain']['iterations']:4d} learned it {o['learned']['iterations']:4d} "
              f"corrected it {c['iterations']:4d} used {c['used_learned_correction']} "
              f"reduction {c['correction_reduction'][0]:.3f} -> {c['correction_reduction'][1]:.3f}")
        assert c["converged"] == 1 and o["learned"]["converged"] == 1
        if c["used_learned_correction"]:
            assert c["correction_reduction"][1] < 0.99 * c["correction_reduction"][0]
    for o in out[:train]:
        assert o["corrected"]["used_learned_correction"] == 0  # weight 0 while training
    for o in out[train:]:
        assert o["corrected"]["correction_reduction"][0] >= 0  # tried on every solve after training
    print("correction held-out explained", np.round(corr.heldout, 3).tolist())


def test_learned_correction_falls_back(cuda, product_lib):
    """An untrained network's correction is a direction unrelated to the residual: even at
    its least-squares scale it lowers the first step's residual by far less than the 1 %
    a correction must gain, so the solve falls back to the plain preconditioner and
    reaches the solution of a solve without any correction."""
    from conductorrigid_b200.device import Handle
    from conductorrigid_b200.learned import Network

    s = systems_small(0.20)
    ref = Handle(_params(s), s.L)
    ref.set_topology(s.body, s.rigid, s.body_charge)
    q0 = ref.dev(np.zeros(s.n_beads))
    p0 = ref.dev(np.zeros(s.n_bodies))
    ref.compute(s.pos, s.body_pos, q0, p0)
    net = Network(seed=11)
    h = Handle(_params(s), s.L)
    h.set_topology(s.body, s.rigid, s.body_charge)
    h.set_correction(net, 1000.0)
    q = h.dev(np.zeros(s.n_beads))
    phi = h.dev(np.zeros(s.n_bodies))
    _, st = h.compute(s.pos, s.body_pos, q, phi)
    print("reductions plain / corrected:", st["correction_reduction"])
    assert st["used_learned_correction"] == 0
    assert 0.99 * st["correction_reduction"][0] <= st["correction_reduction"][1] <= st["correction_reduction"][0]
    assert st["converged"] == 1
    assert float((q - q0).abs().max() / q0.abs().max()) < 1e-5
    h.set_correction(None)
    ref.close()
    h.close()
    net.close()
