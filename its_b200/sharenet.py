"""The share network: data generation, training and evaluation on the GPU.

The exact start (its_exact_start) solves the shell system in one pass for any choice of
the "shares" -- the coefficients of the corner vertices that coincide with a coarser
corner. The reference's solution (Eigen's CGLS from zero, ThinShells.cpp:615-617) is the
minimum-norm one; its shares are what the network learns to predict from 64 local
features (its_share_features), so that the learned start lands next to it.

Training data are the method's own fits: meshes of the uneven multi-mesh mix
(meshes.batch_meshes), each fitted by the FP64 LSCG from zero to a 1e-12 relative
residual; the targets are that solution at the coincident vertices. Training runs on the
GPU through libits' own kernels (its_mlp_train: tcgen05 BF16 GEMMs, Adam).

    python -m its_b200.sharenet train [--meshes 512] [--steps 20000] [--out FILE]
    python -m its_b200.sharenet eval  [--meshes 64]

The trained parameters ship as share_net.f32 beside this file: its_mlp_num_params() FP32
values followed by 130 normalisation values (feature mean[64], feature scale[64], target
mean, target scale).
"""
import argparse
import json
import math
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "share_net.f32")
N_IN, N_HID = 64, 128
NUM_PARAMS = N_HID * N_IN + N_HID + 2 * (N_HID * N_HID + N_HID) + N_HID + 1
NUM_NORM = 2 * N_IN + 2


def init_params(seed=0):
    """Fan-in scaled uniform weights, zero biases (flat layout of its_mlp)."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_out, fan_in in [(N_HID, N_IN), (N_HID, N_HID), (N_HID, N_HID)]:
        parts += [rng.uniform(-1, 1, fan_out * fan_in) * math.sqrt(3.0 / fan_in), np.zeros(fan_out)]
    parts += [rng.uniform(-1, 1, N_HID) * math.sqrt(3.0 / N_HID), np.zeros(1)]
    p = np.concatenate(parts).astype(np.float32)
    assert p.shape[0] == NUM_PARAMS
    return p


def save(path, params, norm):
    np.concatenate([np.asarray(params, np.float32), np.asarray(norm, np.float32)]).astype("<f4").tofile(path)


def load(path=WEIGHTS):
    a = np.fromfile(path, dtype="<f4")
    assert a.shape[0] == NUM_PARAMS + NUM_NORM, "unexpected share network file size"
    return a[:NUM_PARAMS].copy(), a[NUM_PARAMS:].copy()


def prepare(ctx, mesh):
    """Octree and right-hand side of one mesh of the mix (dict from meshes.batch_meshes)."""
    from . import Svo, model_to_unit_cube, uniform_bbox
    V = model_to_unit_cube(mesh["V"])
    o, _, w = uniform_bbox(V)
    svo = Svo(ctx, V, mesh["F"], mesh["res"], o, w)
    b = ctx.signed_distance(svo.vertices()[0], V, mesh["F"])
    return svo, V, b, o, w


def min_norm_fit(svo, b, tol=1e-12):
    """The reference's solution: FP64 LSCG from zero to a tight relative residual."""
    from . import STOP_RESIDUAL, Operator
    op = Operator(svo)
    x, rep = op.solve(b, tol=tol, max_iters=20000, stop_rule=STOP_RESIDUAL)
    op.close()
    return x, rep


def dataset(ctx, meshes, log=None):
    """Raw features and min-norm targets of the coincident vertices of every mesh."""
    feats, targets = [], []
    for k, m in enumerate(meshes):
        svo, V, b, _, _ = prepare(ctx, m)
        x, rep = min_norm_fit(svo, b)
        f, ids = svo.share_features(b)
        feats.append(f)
        targets.append(x[ids].astype(np.float32))
        svo.close()
        if log and (k % 64 == 0 or k == len(meshes) - 1):
            log("mesh %d/%d: %d rows, %d iterations" % (k + 1, len(meshes), f.shape[0], rep["iterations"]))
    return np.concatenate(feats), np.concatenate(targets)


def normalisation(X, y):
    mean = X.mean(0)
    std = X.std(0)
    scale = np.where(std > 1e-12, 1.0 / np.maximum(std, 1e-12), 1.0)
    ym, ys = float(y.mean()), float(y.std()) or 1.0
    return np.concatenate([mean, scale, [ym, ys]]).astype(np.float32)


def train(meshes=512, steps=20000, batch=65536, lr=1e-3, seed=1000, out=WEIGHTS, log=print):
    import torch

    from . import Context, meshes as M
    from .api import ShareNet
    ctx = Context(0)
    t0 = time.time()
    X, y = dataset(ctx, M.batch_meshes(meshes, seed), log)
    log("dataset: %d rows in %.1f s" % (X.shape[0], time.time() - t0))
    norm = normalisation(X, y)
    Xn = ((X - norm[:N_IN]) * norm[N_IN:2 * N_IN]).astype(np.float32)
    yn = ((y - norm[2 * N_IN]) / norm[2 * N_IN + 1]).astype(np.float32)
    Xd, yd = torch.from_numpy(Xn).cuda(), torch.from_numpy(yn).cuda()
    net = ShareNet(ctx, batch=batch, params=init_params(seed))
    t1 = time.time()
    curve = net.train(Xd, yd, steps, lr=lr, seed=seed)
    torch.cuda.synchronize()
    t_train = time.time() - t1
    log("trained %d steps in %.1f s; loss %.4f -> %.4f" % (steps, t_train, curve[:10].mean(), curve[-100:].mean()))
    save(out, net.params(), norm)
    net.close()
    return dict(rows=int(X.shape[0]), steps=steps, batch=batch, train_s=t_train,
                loss_first=float(curve[:10].mean()), loss_last=float(curve[-100:].mean()))


def evaluate(ctx, net, norm, meshes, grid=64):
    """Field error against the min-norm solution: zero shares versus learned shares."""
    from .api import learned_start_batch
    rows = []
    for m in meshes:
        svo, V, b, o, w = prepare(ctx, m)
        x, rep = min_norm_fit(svo, b)
        zero = svo.exact_start(b)
        learned = learned_start_batch([svo], net, [b], norm)[0]
        g = svo.eval_grid(x, o, w, grid)
        scale = float(np.abs(b).max())
        r = dict(faces=m["faces"], res=m["res"], kind=m["kind"], lscg_iterations=rep["iterations"],
                 residual_learned=svo.residual(b, learned), residual_zero=svo.residual(b, zero))
        for name, lam in (("zero", zero), ("learned", learned)):
            d = svo.eval_grid(lam, o, w, grid) - g
            r["grid_rms_" + name] = float(np.sqrt(np.mean(d * d)) / scale)
            r["grid_max_" + name] = float(np.abs(d).max() / scale)
            r["coef_rel_" + name] = float(np.linalg.norm(lam - x) / np.linalg.norm(x))
        rows.append(r)
        svo.close()
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "eval"])
    ap.add_argument("--meshes", type=int, default=None)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--report", default=None)
    a = ap.parse_args()
    if a.cmd == "train":
        res = train(a.meshes or 512, a.steps, a.batch, a.lr, out=a.out)
    else:
        from . import Context, meshes as M
        from .api import ShareNet
        ctx = Context(0)
        params, norm = load(a.out)
        net = ShareNet(ctx, batch=a.batch, params=params)
        rows = evaluate(ctx, net, norm, M.batch_meshes(a.meshes or 64, 5000))
        keys = [k for k in rows[0] if k.startswith(("grid_", "coef_", "residual_"))]
        res = {k: float(np.mean([r[k] for r in rows])) for k in keys}
        res["meshes"] = len(rows)
        res["rows"] = rows
    print(json.dumps({k: v for k, v in res.items() if k != "rows"}))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
