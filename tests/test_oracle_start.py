"""The oracle's exact start in explicit form (each surplus from G = b - finer shares and
the parent cell's hats) against the sequential coarse-to-fine definition, on the CPU: the
two are the same solution of A lambda = b, to rounding, for zero and for arbitrary shares."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from conftest import prepared_mesh


@pytest.mark.parametrize("name,kw,res", [("small", {}, 16), ("torus", dict(R=0.7, r=0.25, rings=48, segs=24), 32)])
def test_explicit_exact_start_equals_sequential_surplus(name, kw, res):
    V, F, o, w = prepared_mesh(name, **kw)
    ref = oracle.Svo(V, F, res, o, w)
    pos, _ = ref.vertices()
    rng = np.random.default_rng(7)
    # a function of position: coincident vertices (one point) get one value, as the system needs
    b = np.linalg.norm(pos - 0.5, axis=1) - 0.3 + 0.05 * np.sin(7 * pos[:, 0]) * np.cos(5 * pos[:, 1])
    rp, col, val = ref.assemble()
    n = rp.shape[0] - 1
    A = sp.csr_matrix((val, col, rp), shape=(n, n))
    for shares in (None, rng.standard_normal(n)):
        lam = ref.exact_start(b, shares)
        seq = ref.exact_start(b, shares, form="surplus")
        assert np.linalg.norm(A @ lam - b) <= 1e-14 * np.linalg.norm(b)
        assert np.linalg.norm(A @ seq - b) <= 1e-14 * np.linalg.norm(b)
        assert np.abs(lam - seq).max() <= 1e-12 * np.abs(seq).max()
        if shares is not None:  # the shares are kept where they apply, identically in both
            kept = lam == shares
            assert np.array_equal(kept, seq == shares) and kept.any()
