"""Failure detection on the GPU without a fault: a bounded device wait that runs out.

The tensor-core network kernels wait on an mbarrier for their MMAs, each wait bounded
by a clock-cycle limit.  Here the limit is made short and the next launch withholds its
first MMAs and their commit, so nothing ever arrives on the barrier: every CTA's wait
runs out, the CTA frees its tensor memory and exits, and the call returns CR_TIMEOUT.
Nothing is left in flight, so the network and the CUDA context stay usable: the next
calls reproduce the results from before."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_mlp_wait_runs_out_and_network_stays_usable(cuda, product_lib):
    from conductorrigid_b200._lib import CrError
    from conductorrigid_b200.learned import FEATURES, Network

    torch = cuda
    net = Network(seed=5)
    g = torch.Generator(device="cuda").manual_seed(3)
    n = 3000
    x = torch.randn(n, FEATURES, device="cuda", generator=g).to(torch.bfloat16).view(torch.int16).contiguous()
    t = torch.randn(n, device="cuda", generator=g)
    y0 = net.forward(x).cpu().numpy()

    # forward: the wait runs out
    net.set_wait(200_000, withhold_next=True)
    with pytest.raises(CrError) as e:
        net.forward(x)
    assert e.value.status == product_lib.CR_TIMEOUT
    assert "ran out" in str(e.value)
    # training: the same, and no gradient is accumulated
    net.set_wait(200_000, withhold_next=True)
    with pytest.raises(CrError) as e:
        net.accumulate_grad(x, t)
    assert e.value.status == product_lib.CR_TIMEOUT
    assert np.abs(net.grads()).max() == 0.0

    # the default limit again: the network works and gives the same outputs as before
    net.set_wait()
    y1 = net.forward(x).cpu().numpy()
    assert np.array_equal(y0, y1)
    loss = net.train_step(x, t)
    assert np.isfinite(loss) and loss > 0
    net.close()


def test_realspace_wait_runs_out_and_handle_stays_usable(cuda, product_lib):
    """The streamed real-space product (CR_REALSPACE_STREAM): with the copies of the next
    product withheld, every consumer warp's first wait runs out, the call returns
    CR_TIMEOUT, and the next products (default limit) reproduce the results from before."""
    from conductorrigid_b200 import _lib, systems
    from conductorrigid_b200._lib import CrError
    from conductorrigid_b200.device import Handle

    torch = cuda
    s = systems.spheres(np.ones(40), 2, 0.30, (0.0, 0.0, 1.0), seed=11)
    h = Handle(_lib.make_params(xi=systems.XI_DEFAULT, errortol=1e-5, grid=32, support=9, rcut=4.0,
                                field=tuple(s.field), precision="mixed", precond="conductor"), s.L)
    h.set_topology(s.body, s.rigid, s.body_charge)
    h.set_realspace(_lib.CR_REALSPACE_STREAM)
    h.set_positions(s.pos, s.body_pos)
    g = torch.Generator(device="cpu").manual_seed(2)
    x = torch.randn(s.n_beads + s.n_bodies, dtype=torch.float64, generator=g).cuda()
    y32 = h.apply_operator(x, _lib.CR_FP32).cpu().numpy()
    y64 = h.apply_operator(x, _lib.CR_FP64).cpu().numpy()
    for prec in (_lib.CR_FP32, _lib.CR_FP64):
        h.set_wait_limit(200_000, withhold_next=True)
        with pytest.raises(CrError) as e:
            h.apply_operator(x, prec)
        assert e.value.status == product_lib.CR_TIMEOUT
        assert "ran out" in str(e.value)
    h.set_wait_limit()
    z32 = h.apply_operator(x, _lib.CR_FP32).cpu().numpy()
    z64 = h.apply_operator(x, _lib.CR_FP64).cpu().numpy()
    # the per-cluster sums are added with atomics: equal up to the order of the additions
    assert np.linalg.norm(z32 - y32) <= 1e-6 * np.linalg.norm(y32)
    assert np.linalg.norm(z64 - y64) <= 1e-13 * np.linalg.norm(y64)
    h.close()
