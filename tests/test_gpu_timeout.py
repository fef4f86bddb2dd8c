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
