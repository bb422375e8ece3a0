"""Learned start: share-network features against the numpy oracle, and the learned start
as the composition features -> network -> exact start.

Bars: features agree with the oracle to FP32 rounding (1e-5 relative per feature, the FP64
sums being formed in the same order); the learned start equals the exact start with the
network's shares bit for bit and has a residual at rounding level.
"""
import numpy as np
import pytest

import oracle
from conftest import prepared_mesh
from oracle import features as ofeat
from oracle import mlp as omlp

CASES = [("small", {}, 16), ("c0", {}, 32), ("torus", dict(R=0.7, r=0.25, rings=48, segs=24), 32)]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,res", CASES, ids=[f"{c[0]}-{c[2]}" for c in CASES])
def test_share_features_match_oracle(ctx, name, kw, res):
    from its_b200 import Svo
    V, F, o, w = prepared_mesh(name, **kw)
    ref = oracle.Svo(V, F, res, o, w)
    gpu = Svo(ctx, V, F, res, o, w)
    b = oracle.signed_distance(ref.vertices()[0], V, F)
    lam0 = ref.exact_start(b)
    f_ref, ids_ref = ofeat.share_features(ref, b, V, F, lam0)
    f_gpu, ids_gpu = gpu.share_features(b)
    assert np.array_equal(ids_gpu, ids_ref) and len(ids_ref) > 0
    scale = np.maximum(np.abs(f_ref).max(0), 1e-30)
    err = (np.abs(f_gpu - f_ref) / scale).max(0)
    assert err.max() <= 1e-5, np.argmax(err)
    # normalisation is (f - mean) * scale
    rng = np.random.default_rng(0)
    norm = np.concatenate([rng.standard_normal(64), rng.uniform(0.5, 2, 64)]).astype(np.float32)
    f_n, _ = gpu.share_features(b, norm)
    assert np.allclose(f_n, (f_gpu - norm[:64]) * norm[64:], rtol=1e-6, atol=1e-6)


@pytest.mark.gpu
def test_learned_start_is_exact_start_with_predicted_shares(ctx):
    from its_b200 import Svo
    from its_b200.api import ShareNet, learned_start_batch
    net = ShareNet(ctx, batch=4096, params=omlp.init_params(7) * np.float32(0.1))
    rng = np.random.default_rng(1)
    norm = np.concatenate([rng.standard_normal(64) * 0.01, np.ones(64), [0.001, 0.01]]).astype(np.float32)
    svos, bs, meshes = [], [], []
    for name, kw, res in CASES:
        V, F, o, w = prepared_mesh(name, **kw)
        s = Svo(ctx, V, F, res, o, w)
        svos.append(s)
        bs.append(ctx.signed_distance(s.vertices()[0], V, F))
        meshes.append((V, F))
    outs = learned_start_batch(svos, net, bs, norm)
    for s, b, (V, F), lam in zip(svos, bs, meshes, outs):
        feats, ids = s.share_features(b, norm[:128])
        shares = np.zeros(s.num_verts)
        shares[ids] = net.forward(feats).astype(np.float64) * float(norm[129]) + float(norm[128])
        assert np.array_equal(lam, s.exact_start(b, shares))
        assert s.residual(b, lam) <= 1e-14
    net.close()


@pytest.mark.gpu
def test_trained_network_gain_on_held_out_meshes(ctx):
    # What the trained network gains over the method without it, on held-out meshes of the
    # uneven mix (seeds never seen in training): the plain LSCG needs tens of iterations to
    # reach 1e-6; the learned start is exact at once (residual at rounding level), and its
    # field is much closer to the minimum-norm (reference) solution than the zero-share start.
    from its_b200 import meshes, sharenet
    from its_b200.api import ShareNet, learned_start_batch
    params, norm = sharenet.load()
    net = ShareNet(ctx, batch=65536, params=params)
    mix = sorted(meshes.batch_meshes(64, 5000), key=lambda m: m["faces"])[:6]
    err = {"zero": [], "learned": []}
    for m in mix:
        svo, V, b, o, w = sharenet.prepare(ctx, m)
        x, rep = sharenet.min_norm_fit(svo, b)
        from its_b200 import STOP_RESIDUAL, Operator
        op = Operator(svo)
        _, plain = op.solve(b, tol=1e-6, stop_rule=STOP_RESIDUAL)
        op.close()
        learned = learned_start_batch([svo], net, [b], norm)[0]
        zero = svo.exact_start(b)
        assert svo.residual(b, learned) <= 1e-13 and plain["iterations"] >= 10
        g = svo.eval_grid(x, o, w, 48)
        for name, lam in (("zero", zero), ("learned", learned)):
            d = svo.eval_grid(lam, o, w, 48) - g
            err[name].append(np.sqrt(np.mean(d * d)) / np.abs(b).max())
        svo.close()
    assert np.mean(err["learned"]) <= 0.25 * np.mean(err["zero"]), err
    net.close()


@pytest.mark.gpu
def test_learned_fit_graph_equals_start_and_check(ctx):
    # its_learned_fit (captured once, then replayed) gives the learned start bit for bit and
    # the matrix-free residual; new values of b are read at every replay, new addresses
    # re-capture, host vectors are staged; a tolerance below the start's residual runs the
    # plain LSCG from the start
    import torch
    from its_b200 import Svo
    from its_b200.api import ShareNet, learned_fit, learned_start_batch
    net = ShareNet(ctx, batch=4096, params=omlp.init_params(7) * np.float32(0.1))
    rng = np.random.default_rng(1)
    norm = np.concatenate([rng.standard_normal(64) * 0.01, np.ones(64), [0.001, 0.01]]).astype(np.float32)
    V, F, o, w = prepared_mesh("torus", R=0.7, r=0.25, rings=48, segs=24)
    s = Svo(ctx, V, F, 32, o, w)
    b = ctx.signed_distance(s.vertices()[0], V, F)
    ref = learned_start_batch([s], net, [b], norm)[0]
    b_dev = torch.from_numpy(b).cuda()
    lam_dev = torch.empty_like(b_dev)
    for _ in range(3):
        lam_dev.zero_()
        _, rep = learned_fit(s, net, b_dev, norm, 1e-6, out=lam_dev)
        assert np.array_equal(lam_dev.cpu().numpy(), ref)
        assert rep["iterations"] == 0 and rep["converged"] and rep["rel_residual"] == s.residual(b, ref)
    b_dev.mul_(0.5)  # same address, new values
    learned_fit(s, net, b_dev, norm, 1e-6, out=lam_dev)
    assert np.array_equal(lam_dev.cpu().numpy(), learned_start_batch([s], net, [0.5 * b], norm)[0])
    lam_host, rep = learned_fit(s, net, b, norm, 1e-6)  # host vectors
    assert np.array_equal(lam_host, ref) and rep["iterations"] == 0
    b_pin = torch.from_numpy(b).pin_memory()  # page-locked host vectors: copied by the graph
    lam_pin = torch.zeros(s.num_verts, dtype=torch.float64).pin_memory()
    for k in range(2):
        lam_pin.zero_()
        learned_fit(s, net, b_pin.numpy(), norm, 1e-6, out=lam_pin.numpy())
        assert np.array_equal(lam_pin.numpy(), ref)
    norm2 = norm.copy()
    norm2[128] += 0.001  # another normalisation: another graph
    lam2, _ = learned_fit(s, net, b, norm2, 1e-6)
    assert np.array_equal(lam2, learned_start_batch([s], net, [b], norm2)[0])
    x, rep = learned_fit(s, net, b, norm, 0.1 * rep["rel_residual"])
    assert rep["iterations"] > 0 and np.isfinite(rep["rel_residual"])
    net.close()
    # another network (perhaps at the freed one's address): captured anew
    net2 = ShareNet(ctx, batch=4096, params=omlp.init_params(9) * np.float32(0.1))
    lam3, _ = learned_fit(s, net2, b, norm, 1e-6)
    assert np.array_equal(lam3, learned_start_batch([s], net2, [b], norm)[0])
    net2.close()


@pytest.mark.gpu
def test_tuned_fit_launches_change_speed_not_bits():
    # with tuning on, the exact start's block size is measured (before the learned fit's graph
    # is captured) and kept; the start, the learned fit and the batched start are the untuned
    # ones bit for bit
    import torch
    from its_b200 import Context, Svo
    from its_b200.api import ShareNet, learned_fit, learned_start_batch
    rng = np.random.default_rng(1)
    norm = np.concatenate([rng.standard_normal(64) * 0.01, np.ones(64), [0.001, 0.01]]).astype(np.float32)
    V, F, o, w = prepared_mesh("torus", R=0.7, r=0.25, rings=48, segs=24)
    outs = []
    for tuned in (False, True):
        ctx = Context(0)
        if tuned:
            ctx.set_autotune(True)
        net = ShareNet(ctx, batch=4096, params=omlp.init_params(7) * np.float32(0.1))
        s = Svo(ctx, V, F, 32, o, w)
        b = ctx.signed_distance(s.vertices()[0], V, F)
        zero = s.exact_start(b)
        start = learned_start_batch([s], net, [b], norm)[0]
        b_dev = torch.from_numpy(b).cuda()
        lam_dev = torch.zeros_like(b_dev)
        learned_fit(s, net, b_dev, norm, 1e-6, out=lam_dev)
        learned_fit(s, net, b_dev, norm, 1e-6, out=lam_dev)  # the replay
        outs.append((zero, start, lam_dev.cpu().numpy(), ctx.autotune_choices()))
        net.close()
        s.close()
        ctx.close()
    for a, b_ in zip(outs[0][:3], outs[1][:3]):
        assert np.array_equal(a, b_)
    assert any(k.startswith("exact_start/") for k in outs[1][3])
