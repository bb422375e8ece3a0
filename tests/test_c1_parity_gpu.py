"""Parity on the benchmark's own workload: the (3,5) torus-knot tube, 1,048,576 faces, SVO
depth 9 (res 256), marching cubes at 512^3.

Bars:
  * octree, occupancy, neighbours, corner vertices and fine edges: bit-exact with the oracle;
  * shell samples (edge and face intersections): the same point set as the oracle's;
  * right-hand side: distances bit-exact with the oracle's BVH signed distance, and the same
    signs (both take the sign from the same fast winding number over the same tree);
  * the 513^3 FP64 lattice field of the FP64 LSCG fit: bit-exact with the oracle's, and the
    512^3 marching-cubes case indices at both shell iso levels bit-exact with the oracle's;
  * the learned fit (its_learned_fit, the benchmark's step): every case index at both shell
    iso levels equal to those of the FP64 LSCG from zero at 1e-12 (the solution the
    reference's LSCG converges to, ThinShells.cpp:615-617) -- the learned fit's field differs
    from it only in coarse cells away from the surface.
"""
import numpy as np
import pytest

import oracle

R_MC = 512


@pytest.fixture(scope="module")
def c1(ctx):
    import its_b200
    from its_b200 import Svo, meshes
    V, F = meshes.config_mesh("c1")
    V = its_b200.model_to_unit_cube(V)
    o, _, w = its_b200.uniform_bbox(V)
    gpu = Svo(ctx, V, F, 256, o, w)
    ref = oracle.Svo(V, F, 256, o, w)
    yield V, F, o, w, gpu, ref
    gpu.close()


@pytest.mark.gpu
def test_c1_octree_bit_exact(c1):
    V, F, o, w, gpu, ref = c1
    assert gpu.depth == ref.depth == 9
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
    assert np.array_equal(go, ro) and np.array_equal(gp, rp)
    for a, b in zip(gpu.edges(), ref.edges()):
        assert np.array_equal(a, b)


@pytest.mark.gpu
def test_c1_shell_samples_same_point_set(c1):
    # edge and face intersections (ThinShells::cpIntersectionPoints): the same points, the
    # same split between the two kinds; the GPU emits them in mesh order, the oracle in the
    # reference's sweep order
    V, F, o, w, gpu, ref = c1
    pts_ref, ne_ref = ref.intersections()
    pts_gpu, ne_gpu = gpu.shell_samples(V, F)
    assert ne_gpu == ne_ref and len(pts_gpu) == len(pts_ref)
    key = lambda P: P[np.lexsort((P[:, 2], P[:, 1], P[:, 0]))]  # noqa: E731
    assert np.array_equal(key(pts_gpu[:ne_gpu]), key(pts_ref[:ne_ref]))
    assert np.array_equal(key(pts_gpu[ne_gpu:]), key(pts_ref[ne_ref:]))


@pytest.mark.gpu
def test_c1_signed_distance_matches_oracle(ctx, c1):
    V, F, o, w, gpu, ref = c1
    pos, _ = gpu.vertices()
    b = ctx.signed_distance(pos, V, F)
    b_ref = oracle.signed_distance_bvh(pos, V, F)
    assert np.array_equal(np.abs(b), np.abs(b_ref))
    assert np.array_equal(np.signbit(b), np.signbit(b_ref))


@pytest.fixture(scope="module")
def c1_fit(ctx, c1):
    from its_b200 import STOP_RESIDUAL, Operator
    V, F, o, w, gpu, ref = c1
    pos, _ = gpu.vertices()
    b = ctx.signed_distance(pos, V, F)
    op = Operator(gpu)
    lam, rep = op.solve(b, tol=1e-6, stop_rule=STOP_RESIDUAL)
    lam_ref, rep_ref = op.solve(b, tol=1e-12, max_iters=20000, stop_rule=STOP_RESIDUAL)
    op.close()
    assert rep["converged"] and rep_ref["converged"]
    pts, _ = gpu.shell_samples(V, F)
    inner, outer, _ = gpu.shell_iso_values(lam_ref, np.vstack([V, pts]))
    return b, lam, lam_ref, inner, outer


@pytest.mark.gpu
def test_c1_field_and_marching_cubes_bit_exact(ctx, c1, c1_fit):
    V, F, o, w, gpu, ref = c1
    b, lam, lam_ref, inner, outer = c1_fit
    field = gpu.eval_grid(lam, o, w, R_MC)
    field_ref = ref.eval_grid(lam, o, w, R_MC)
    assert np.array_equal(field, field_ref)
    del field_ref
    for iso in (inner, outer):
        cube, _, n = ctx.marching_cubes(field, R_MC, o, w, iso, triangles=False)
        cube_ref, _, n_ref = oracle.marching_cubes(field, R_MC, o, w, iso, with_triangles=False)
        assert n == n_ref and np.array_equal(cube, cube_ref)


@pytest.mark.gpu
def test_c1_learned_fit_keeps_mc_topology(ctx, c1, c1_fit):
    import torch
    from its_b200 import sharenet
    from its_b200.api import ShareNet, learned_fit
    V, F, o, w, gpu, ref = c1
    b, lam, lam_ref, inner, outer = c1_fit
    params, norm = sharenet.load()
    net = ShareNet(ctx, batch=65536, params=params)
    try:
        lam_l, rep = learned_fit(gpu, net, b, norm, 1e-6)
    finally:
        net.close()
    assert rep["rel_residual"] <= 1e-6
    M = R_MC + 1
    fa = torch.empty(M ** 3, dtype=torch.float64, device="cuda")
    fb = torch.empty_like(fa)
    gpu.eval_grid(lam_l, o, w, R_MC, out=fa)
    gpu.eval_grid(lam_ref, o, w, R_MC, out=fb)
    for iso in (inner, outer):
        ca, _, na = ctx.marching_cubes(fa, R_MC, o, w, iso, triangles=False)
        cb, _, nb = ctx.marching_cubes(fb, R_MC, o, w, iso, triangles=False)
        assert np.count_nonzero(ca != cb) == 0 and na == nb
