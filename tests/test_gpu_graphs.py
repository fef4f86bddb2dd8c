"""Captured Arnoldi steps (CUDA graphs): the same iterations and solutions as the
uncaptured loop, re-captured for a new geometry, off under the profiler and without a
stream, and in batched solves."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system():
    from conductorrigid_b200 import systems

    return systems.workload("plain_small", scale=0.3).system


def _solve(s, graphs, stream, **kw):
    import torch

    from conductorrigid_b200 import _lib
    from conductorrigid_b200.device import Handle

    P = _lib.make_params(field=tuple(s.field), xi=0.85, errortol=1e-5, grid=48, support=9, rcut=4.0, gmres_tol=1e-6,
                         maxiter=4000, **kw)
    h = Handle(P, s.L, stream=stream)
    h.set_graphs(graphs)
    h.set_topology(s.body, s.rigid, s.body_charge)
    out = []
    with torch.cuda.stream(stream) if stream is not None else torch.cuda.stream(torch.cuda.current_stream()):
        for pos in (s.pos, s.pos + 0.01):  # a second geometry: the graph is captured again
            q = torch.zeros(s.n_beads, dtype=torch.float64, device="cuda")
            phi = torch.zeros(s.n_bodies, dtype=torch.float64, device="cuda")
            F, st = h.compute(pos, s.body_pos + 0.01 * (pos is not s.pos), q, phi)
            torch.cuda.synchronize()
            out.append((q.cpu().numpy(), phi.cpu().numpy(), F.cpu().numpy(), st))
    n_graph = h.graph_launches()
    h.close()
    return out, n_graph


@pytest.mark.parametrize("kw", [dict(precision="mixed", precond="conductor", restart=20),
                                dict(precision="fp64", precond="conductor", restart=20),
                                dict(precision="fp64", precond="diagonal", restart=30)])
def test_graph_steps_match_uncaptured(cuda, product_lib, kw):
    torch = cuda
    s = _system()
    stream = torch.cuda.Stream()
    eager, n0 = _solve(s, False, stream, **kw)
    graph, n1 = _solve(s, True, stream, **kw)
    assert n0 == 0 and n1 > 0
    for (qa, pa, Fa, sa), (qb, pb, Fb, sb) in zip(eager, graph):
        assert sb["converged"] == 1 and sb["final_residual"] <= 1e-6
        assert abs(sa["iterations"] - sb["iterations"]) <= 1
        for a, b in ((qa, qb), (pa, pb), (Fa, Fb)):
            assert np.abs(a - b).max() <= 1e-6 * np.abs(a).max()
    assert n1 >= sum(o[3]["iterations"] for o in graph)


def test_graphs_off_without_stream_and_under_profiler(cuda, product_lib):
    from conductorrigid_b200 import _lib
    from conductorrigid_b200.device import Handle

    torch = cuda
    s = _system()
    P = _lib.make_params(field=tuple(s.field), xi=0.85, errortol=1e-5, grid=48, support=9, rcut=4.0, gmres_tol=1e-6,
                         maxiter=4000, precision="mixed", precond="conductor", restart=20)
    h = Handle(P, s.L)  # legacy default stream: nothing to capture on
    h.set_topology(s.body, s.rigid, s.body_charge)
    q = h.dev(np.zeros(s.n_beads))
    phi = h.dev(np.zeros(s.n_bodies))
    h.compute(s.pos, s.body_pos, q, phi)
    assert h.graph_launches() == 0
    h.close()
    stream = torch.cuda.Stream()
    h = Handle(P, s.L, stream=stream)
    h.set_topology(s.body, s.rigid, s.body_charge)
    h.profile(True)
    with torch.cuda.stream(stream):
        q.zero_()
        phi.zero_()
        h.compute(s.pos, s.body_pos, q, phi)
    torch.cuda.synchronize()
    assert h.graph_launches() == 0
    assert h.profile_read()["krylov"]["launches"] > 0
    h.close()
