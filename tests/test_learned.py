"""The per-bead tensor-core network: CPU restatement checked by finite differences, the
tcgen05 forward and backward kernels checked against it on the GPU, and training."""
import numpy as np
import pytest

from oracle import mlp_ref


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = mlp_ref.bf16_bits(rng.standard_normal((n, mlp_ref.F)))
    t = (np.sin(mlp_ref.from_bits(x)[:, 0]) + 0.5 * mlp_ref.from_bits(x)[:, 1] * mlp_ref.from_bits(x)[:, 2])
    return x, t.astype(np.float32)


def _params(seed):
    rng = np.random.default_rng(seed)
    p = np.zeros(mlp_ref.NPARAM)
    p[mlp_ref.OFF_W1:mlp_ref.OFF_B1] = rng.uniform(-1, 1, mlp_ref.H * mlp_ref.F) * np.sqrt(3 / mlp_ref.F)
    p[mlp_ref.OFF_B1:mlp_ref.OFF_W2] = 0.1 * rng.standard_normal(mlp_ref.H)
    p[mlp_ref.OFF_W2:mlp_ref.OFF_B2] = rng.uniform(-1, 1, mlp_ref.H * mlp_ref.H) * np.sqrt(3 / mlp_ref.H)
    p[mlp_ref.OFF_B2:mlp_ref.OFF_W3] = 0.1 * rng.standard_normal(mlp_ref.H)
    p[mlp_ref.OFF_W3:mlp_ref.OFF_B3] = 0.3 * rng.standard_normal(mlp_ref.H)
    p[mlp_ref.OFF_B3] = 0.05
    return p.astype(np.float32)


def test_restatement_gradient_matches_finite_differences():
    x, t = _data(37, 0)
    p = _params(1).astype(np.float64)
    _, g = mlp_ref.loss_and_grad(p, x, t, rounding=False)
    rng = np.random.default_rng(2)
    blocks = [(mlp_ref.OFF_W1, mlp_ref.OFF_B1), (mlp_ref.OFF_B1, mlp_ref.OFF_W2), (mlp_ref.OFF_W2, mlp_ref.OFF_B2),
              (mlp_ref.OFF_B2, mlp_ref.OFF_W3), (mlp_ref.OFF_W3, mlp_ref.OFF_B3), (mlp_ref.OFF_B3, mlp_ref.NPARAM)]
    for lo, hi in blocks:
        for i in rng.integers(lo, hi, size=min(4, hi - lo)):
            e = 1e-6
            pp, pm = p.copy(), p.copy()
            pp[i] += e
            pm[i] -= e
            fd = (mlp_ref.loss_and_grad(pp, x, t, rounding=False)[0] -
                  mlp_ref.loss_and_grad(pm, x, t, rounding=False)[0]) / (2 * e)
            assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-5], dtype=np.float32)
    r = mlp_ref.bf16_round(v)
    assert r[0] == 1.0 and r[1] == 1.0  # exactly halfway: ties to even
    assert r[2] == 1.0078125
    assert r[3] == -2.5
    assert np.array_equal(mlp_ref.from_bits(mlp_ref.bf16_bits(v)), r)


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, dtype=np.float64) - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 300, 1000, 4096])
def test_tensor_core_forward_and_gradients_match_cpu(cuda, product_lib, n):
    from conductorrigid_b200.learned import Network

    net = Network(seed=3)
    p = _params(4)
    net.set_params(p)
    x, t = _data(n, 5)
    y = net.forward(x).cpu().numpy()
    y_ref = mlp_ref.forward(p, x)
    assert _rel(y, y_ref) < 2e-3
    loss = net.accumulate_grad(x, t)
    g = net.grads()
    loss_ref, g_ref = mlp_ref.loss_and_grad(p, x, t)
    assert abs(loss - loss_ref) <= 2e-3 * loss_ref
    names = ["W1", "b1", "W2", "b2", "w3", "b3"]
    offs = [mlp_ref.OFF_W1, mlp_ref.OFF_B1, mlp_ref.OFF_W2, mlp_ref.OFF_B2, mlp_ref.OFF_W3, mlp_ref.OFF_B3,
            mlp_ref.NPARAM]
    for k, name in enumerate(names):
        lo, hi = offs[k], offs[k + 1]
        assert _rel(g[lo:hi], g_ref[lo:hi]) < 5e-3, (name, _rel(g[lo:hi], g_ref[lo:hi]))
    # a second accumulation doubles the buffer; the optimiser step clears it
    net.accumulate_grad(x, t)
    assert _rel(net.grads(), 2 * g_ref) < 5e-3
    net.adam(1e-3)
    assert not np.any(net.grads())
    net.close()


@pytest.mark.gpu
def test_tensor_core_training_reduces_loss(cuda, product_lib):
    from conductorrigid_b200.learned import Network

    net = Network(seed=7)
    x, t = _data(20000, 8)
    first = net.train_step(x, t, lr=3e-3)
    for _ in range(300):
        last = net.train_step(x, t, lr=3e-3)
    assert last < 0.1 * first, (first, last)
    c = net.counters()
    assert c["adam_steps"] == 301 and c["kernel_launches"] == 602
    net.close()
