"""Share network (tcgen05 BF16 GEMMs, FP32 accumulation) against the numpy oracle.

Bars: the forward pass matches the oracle's BF16-emulating forward to 1e-2 of the output
scale (the kernels sum in FP32 in another order, so a hidden activation can round to the
neighbouring BF16 value); each parameter block's gradient matches to 2e-2 relative
(Frobenius); training lowers the loss and is bit-for-bit repeatable.
"""
import numpy as np
import pytest

from oracle import mlp as ref


def _data(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, ref.N_IN)).astype(np.float32)
    y = (np.sin(X[:, 0]) + 0.5 * X[:, 1] * X[:, 2] - 0.3 * X[:, 3] ** 2).astype(np.float32)
    return X, y


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1000, 70000])
def test_forward_matches_oracle(ctx, n):
    from its_b200.api import ShareNet
    net = ShareNet(ctx, batch=65536, params=ref.init_params(3))
    X, _ = _data(n, 1)
    out = net.forward(X)
    # the fused persistent kernel and the layer-by-layer training kernels agree bit for bit
    assert np.array_equal(out, net.forward_layers(X))
    want = ref.forward(ref.init_params(3), X)
    scale = np.abs(want).max()
    assert np.abs(out - want).max() <= 1e-2 * scale, np.abs(out - want).max() / scale
    net.close()


@pytest.mark.gpu
def test_forward_from_tiles_matches_forward(ctx):
    # the input in the kernel's own tile form (as the learned fit's features kernel writes it)
    # gives the predictions of the FP32-feature path bit for bit, launched as a dependent
    # launch or not
    import torch
    from its_b200.api import ShareNet, feature_tiles
    net = ShareNet(ctx, batch=65536, params=ref.init_params(3))
    X, _ = _data(33505, 4)
    want = net.forward(X)
    tiles = torch.from_numpy(feature_tiles(X)).cuda()
    out = torch.zeros(len(X), dtype=torch.float32, device="cuda")
    net.forward_tiles_async(tiles, len(X), out)
    net.forward_tiles_async(tiles, len(X), out, after_kernel=True)
    net.check()
    assert np.array_equal(out.cpu().numpy(), want)
    net.close()


@pytest.mark.gpu
def test_gradient_matches_oracle(ctx):
    from its_b200.api import ShareNet
    P = ref.init_params(4)
    net = ShareNet(ctx, batch=8192, params=P)
    X, y = _data(4096, 2)
    g, loss = net.gradient(X, y)
    g_ref, loss_ref = ref.gradient(P, X, y)
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref
    k = 0
    for name, shape in ref.SHAPES:
        m = int(np.prod(shape))
        a, b = g[k:k + m], g_ref[k:k + m]
        assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b) + 1e-7, (name, np.linalg.norm(a - b) / np.linalg.norm(b))
        k += m
    net.close()


@pytest.mark.gpu
def test_training_lowers_loss_and_repeats(ctx):
    from its_b200.api import ShareNet
    X, y = _data(100000, 3)
    runs = []
    for _ in range(2):
        net = ShareNet(ctx, batch=4096, params=ref.init_params(5))
        curve = net.train(X, y, steps=300, lr=1e-3, seed=11)
        runs.append((curve, net.params()))
        net.close()
    curve = runs[0][0]
    assert curve[-20:].mean() < 0.2 * curve[:5].mean()
    assert np.array_equal(runs[0][1], runs[1][1]) and np.array_equal(runs[0][0], runs[1][0])
