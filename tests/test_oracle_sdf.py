"""The oracle's accelerated signed distance (linear BVH, exact distance, fast winding number;
the restatement that the benchmark's reference arm and the c1 parity tests use) against its
brute-force form (exact distance over every triangle, exact winding number): the same
distances bit for bit and the same signs at the corner vertices of the octree."""
import numpy as np
import pytest

import oracle
from conftest import prepared_mesh


@pytest.mark.parametrize("name,kw,res", [("c0", {}, 32), ("small", {}, 16),
                                         ("torus", dict(R=0.7, r=0.25, rings=48, segs=24), 32)])
def test_bvh_signed_distance_matches_brute_force(name, kw, res):
    V, F, o, w = prepared_mesh(name, **kw)
    pos, _ = oracle.Svo(V, F, res, o, w).vertices()
    exact = oracle.signed_distance(pos, V, F)
    fast = oracle.signed_distance_bvh(pos, V, F)
    assert np.array_equal(np.abs(fast), np.abs(exact))
    assert np.array_equal(np.signbit(fast), np.signbit(exact))
    # away from the mesh too: points on a coarse lattice of the box
    t = np.linspace(0.0, 1.0, 9)
    P = o + w * np.stack(np.meshgrid(t, t, t, indexing="ij"), -1).reshape(-1, 3)
    a, b = oracle.signed_distance(P, V, F), oracle.signed_distance_bvh(P, V, F)
    assert np.array_equal(np.abs(a), np.abs(b)) and np.array_equal(np.signbit(a), np.signbit(b))


def test_bvh_signed_distance_single_triangle():
    V = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0]])
    F = np.array([[0, 1, 2]], np.int32)
    P = np.array([[0.2, 0.2, 0.5], [2.0, 2.0, -1.0], [0.1, 0.1, 0.0]])
    assert np.array_equal(oracle.signed_distance_bvh(P, V, F), oracle.signed_distance(P, V, F))
