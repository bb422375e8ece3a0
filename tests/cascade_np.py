"""The prolongation cascade of its_eval_grid_fast restated in numpy (test infrastructure):
the dense field on the octree's lattice at res * f points per axis, built coarse to fine with
the hats on the exact lattice points."""
import numpy as np


def cascade_numpy(pos, lam, depth_counts, o, unit, res, f):
    """The prolongation cascade restated in numpy (hats on the exact lattice points)."""
    D = len(depth_counts)
    depth = np.repeat(np.arange(D), depth_counts)
    acc = None
    for d in range(D - 1, -1, -1):
        M = (res >> d) + 1
        A = np.zeros((M, M, M))
        sel = depth == d
        X = np.rint((pos[sel] - o) / (unit * 2 ** d)).astype(int)
        A[X[:, 0], X[:, 1], X[:, 2]] = lam[sel]
        acc = A if acc is None else A + _prolong(acc, 2)
    return acc if f == 1 else _prolong(acc, f)


def _prolong(C, f):
    Mc = C.shape[0]
    idx = np.arange((Mc - 1) * f + 1)
    c0, r = idx // f, idx % f
    c1 = np.minimum(c0 + 1, Mc - 1)
    w1 = r / f
    w0 = 1 - w1
    X = w0[:, None, None] * C[c0] + w1[:, None, None] * C[c1]
    Y = w0[None, :, None] * X[:, c0] + w1[None, :, None] * X[:, c1]
    return w0[None, None, :] * Y[:, :, c0] + w1[None, None, :] * Y[:, :, c1]
