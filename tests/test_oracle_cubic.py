"""The oracle's cubic B-spline basis (test infrastructure for libits' cubic mode): known
values of the uniform cubic B-spline, partition of unity, and the assembled rows equal to the
field at their points."""
import numpy as np
import scipy.sparse as sp

import oracle
from conftest import prepared_mesh


def test_bspline3_known_values_and_partition_of_unity():
    t = np.array([0.0, 0.5, -0.5, 1.0, -1.0, 1.5, 2.0, -2.0, 2.5])
    want = np.array([2 / 3, 23 / 48, 23 / 48, 1 / 6, 1 / 6, 1 / 48, 0.0, 0.0, 0.0])
    assert np.allclose(oracle.bspline3(t), want, atol=1e-16)
    x = np.random.default_rng(0).uniform(-3, 3, 1000)
    assert np.abs(sum(oracle.bspline3(x - k) for k in range(-6, 7)) - 1.0).max() <= 4e-16


def test_cubic_rows_are_the_field_at_their_points():
    V, F, o, w = prepared_mesh("small")
    s = oracle.Svo(V, F, 16, o, w)
    eps = 0.01 * float(np.linalg.norm(V.max(0) - V.min(0)))
    P, T = oracle.offset_samples(V, F, eps)
    rp, col, val = s.cubic_assemble(P)
    n, N = s.num_verts, len(rp) - 1
    assert N == n + len(P) and col.max() < n
    lam = np.random.default_rng(1).standard_normal(n)
    A = sp.csr_matrix((val, col, rp), shape=(N, N))
    y = A @ np.concatenate([lam, np.zeros(N - n)])
    assert np.allclose(y[n:], s.cubic_eval(lam, P), rtol=0, atol=1e-13)
    pos, _ = s.vertices()
    assert np.allclose(y[:n], s.cubic_eval(lam, pos), rtol=0, atol=1e-12)
    # a constant coefficient vector on the root depth alone is constant inside the box
    nd, vd = s.depth_counts()
    lam1 = np.zeros(n)
    lam1[-vd[-1]:] = 1.0
    inner = o + w * np.random.default_rng(2).uniform(0.3, 0.7, (50, 3))
    f = s.cubic_eval(lam1, inner)
    assert f.min() > 0 and f.max() <= 1.0 + 1e-15
