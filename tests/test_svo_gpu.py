"""Octree parity: libits (GPU) against the oracle on the same normalised meshes.
Topology, Morton codes, occupancy, neighbours, vertex/edge order and owners are integer
and must be bit-exact; node origins, widths and corner positions follow the same IEEE
operations on both sides and must be bit-exact too."""
import numpy as np
import pytest

import oracle
from conftest import prepared_mesh

CASES = [
    ("small", {}, 8), ("small", {}, 32), ("c0", {}, 32), ("c0", {}, 64),
    ("torus", dict(R=0.7, r=0.25, rings=48, segs=24), 64),
    ("superquadric", dict(e1=0.4, e2=2.5, subdiv=4), 32),
    ("knot", dict(rings=512, segs=32, tube=0.15), 128),
]


def _build_both(ctx, name, kw, res):
    from its_b200 import Svo
    V, F, o, w = prepared_mesh(name, **kw)
    return V, F, oracle.Svo(V, F, res, o, w), Svo(ctx, V, F, res, o, w)


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,res", CASES, ids=[f"{c[0]}-{c[2]}" for c in CASES])
def test_svo_bit_exact(ctx, name, kw, res):
    V, F, ref, gpu = _build_both(ctx, name, kw, res)
    assert gpu.depth == ref.depth
    assert (gpu.num_voxels, gpu.num_fine, gpu.num_nodes, gpu.num_verts, gpu.num_edges) == \
        (ref.num_voxels, ref.num_fine, ref.num_nodes, ref.num_verts, ref.num_edges)
    for a, b in zip(gpu.depth_counts(), ref.depth_counts()):
        assert np.array_equal(a, b)
    assert np.array_equal(gpu.voxels(), ref.voxels())
    gn, rn = gpu.nodes(), ref.nodes()
    for k in ("morton", "parent", "childs", "is_leaf", "neighbors", "origin", "width"):
        assert np.array_equal(gn[k], rn[k]), k
    gp, go = gpu.vertices()
    rp, ro = ref.vertices()
    assert np.array_equal(go, ro)
    assert np.array_equal(gp, rp)
    ge, re_ = gpu.edges(), ref.edges()
    for a, b in zip(ge, re_):
        assert np.array_equal(a, b)


@pytest.mark.gpu
def test_svo_rejects_bad_input(ctx):
    from its_b200 import ItsError, Svo
    V, F, o, w = prepared_mesh("small")
    with pytest.raises(ItsError):
        Svo(ctx, V, F, 48, o, w)          # not a power of two
    Fb = F.copy()
    Fb[0, 0] = V.shape[0]
    with pytest.raises(ItsError):
        Svo(ctx, V, Fb, 16, o, w)         # face index out of range
    Vb = V.copy()
    Vb[3, 1] = np.nan
    with pytest.raises(ItsError):
        Svo(ctx, Vb, F, 16, o, w)         # non-finite vertex


@pytest.mark.gpu
def test_svo_single_triangle(ctx):
    from its_b200 import Svo
    V = np.array([[0.2, 0.2, 0.3], [0.7, 0.25, 0.35], [0.4, 0.8, 0.6]])
    F = np.array([[0, 1, 2]], np.int32)
    o, e, w = oracle.uniform_bbox(V)
    ref, gpu = oracle.Svo(V, F, 16, o, w), Svo(ctx, V, F, 16, o, w)
    assert gpu.depth == ref.depth and gpu.num_nodes == ref.num_nodes
    assert np.array_equal(gpu.voxels(), ref.voxels())
    assert np.array_equal(gpu.nodes()["neighbors"], ref.nodes()["neighbors"])
    assert np.array_equal(gpu.vertices()[0], ref.vertices()[0])
