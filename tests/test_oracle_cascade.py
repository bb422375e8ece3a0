"""On the CPU: the prolongation cascade (numpy) against the oracle's point-by-point field, the
reference's sums. They differ only by the reference's single-precision geometry (corner
positions and a padded box a few 1e-9 off the lattice), far below FP32 rounding."""
import numpy as np

import oracle
from cascade_np import cascade_numpy
from conftest import prepared_mesh


def test_cascade_matches_reference_field():
    V, F, o, w = prepared_mesh("small")
    res = 16
    ref = oracle.Svo(V, F, res, o, w)
    pos, _ = ref.vertices()
    lam = np.random.default_rng(0).standard_normal(pos.shape[0])
    unit = np.full(3, np.asarray(w, float)[0] / res)
    for f in (1, 2):
        R = res * f
        M = R + 1
        exact = ref.eval_grid(lam, o, w, R).reshape(M, M, M).transpose(2, 1, 0)
        cas = cascade_numpy(pos, lam, ref.depth_counts()[1], np.asarray(o, float), unit, res, f)
        assert np.abs(cas - exact).max() <= 1e-6 * np.abs(exact).max()
