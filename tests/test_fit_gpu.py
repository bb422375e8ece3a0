"""Fit-path parity: libits (GPU) against the oracle on the same inputs.

Bars: the assembled operator (structure and values) is bit-exact; the transpose is exact;
SpMV agrees to 1e-14 relative (different summation order only where rows are binned);
signed distances are bit-exact in magnitude (same IEEE operations, min is order-free) with
the same sign wherever |b| > 1e-9; CGLS follows Eigen's algorithm with GPU tree reductions
instead of sequential dots, so lambda agrees to 1e-8 relative and the iteration count to
within 1; the shell samples are the same point set.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from conftest import prepared_mesh

FIT_CASES = [("small", {}, 16), ("c0", {}, 32), ("torus", dict(R=0.7, r=0.25, rings=48, segs=24), 32)]


def _setup(ctx, name, kw, res):
    from its_b200 import Svo
    V, F, o, w = prepared_mesh(name, **kw)
    return V, F, oracle.Svo(V, F, res, o, w), Svo(ctx, V, F, res, o, w)


@pytest.mark.gpu
def test_tri_attributes_bit_exact(ctx):
    V, F, o, w = prepared_mesh("c0")
    for a, b in zip(ctx.tri_attributes(V, F), oracle.tri_attributes(V, F)):
        assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,res", FIT_CASES, ids=[f"{c[0]}-{c[2]}" for c in FIT_CASES])
def test_operator_bit_exact(ctx, name, kw, res):
    from its_b200 import Operator
    V, F, ref, gpu = _setup(ctx, name, kw, res)
    op = Operator(gpu)
    rp, col, val = op.csr()
    orp, ocol, oval = ref.assemble()
    assert np.array_equal(rp, orp)
    assert np.array_equal(col, ocol)
    assert np.array_equal(val, oval)
    A = sp.csr_matrix((oval, ocol, orp), shape=(op.rows, op.rows))
    x = np.random.default_rng(1).standard_normal(op.rows)
    y, yt = op.apply(x), op.apply(x, transpose=True)
    assert np.allclose(y, A @ x, rtol=1e-14, atol=1e-14 * np.abs(A @ x).max())
    assert np.allclose(yt, A.T @ x, rtol=1e-13, atol=1e-13 * np.abs(A.T @ x).max())


@pytest.mark.gpu
def test_signed_distance_matches_oracle(ctx):
    V, F, o, w = prepared_mesh("c0")
    ref = oracle.Svo(V, F, 16, o, w)
    pos, _ = ref.vertices()
    b_gpu = ctx.signed_distance(pos, V, F)
    b_ref = oracle.signed_distance(pos, V, F)
    assert np.array_equal(np.abs(b_gpu), np.abs(b_ref))
    far = np.abs(b_ref) > 1e-9
    assert np.array_equal(np.sign(b_gpu[far]), np.sign(b_ref[far]))


@pytest.mark.gpu
def test_signed_distance_large_mesh_and_far_points(ctx):
    # BVH pruning must still find the exact nearest triangle; the fast winding number must
    # give the exact winding number's sign away from the surface.
    V, F, o, w = prepared_mesh("knot", rings=768, segs=48, tube=0.1)
    rng = np.random.default_rng(3)
    P = np.vstack([V[rng.choice(len(V), 500)] + rng.normal(0, 2e-3, (500, 3)),
                   o + w * rng.random((1500, 3))])
    b_gpu = ctx.signed_distance(P, V, F)
    b_ref = oracle.signed_distance(P, V, F)
    assert np.array_equal(np.abs(b_gpu), np.abs(b_ref))
    far = np.abs(b_ref) > 1e-9
    assert np.array_equal(np.sign(b_gpu[far]), np.sign(b_ref[far]))
    assert (b_ref < 0).sum() > 50 and (b_ref > 0).sum() > 50


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,res", FIT_CASES, ids=[f"{c[0]}-{c[2]}" for c in FIT_CASES])
def test_lscg_matches_oracle(ctx, name, kw, res):
    from its_b200 import Operator
    V, F, ref, gpu = _setup(ctx, name, kw, res)
    pos, _ = ref.vertices()
    b = oracle.signed_distance(pos, V, F)
    op = Operator(gpu)
    rp, col, val = ref.assemble()
    A = sp.csr_matrix((val, col, rp), shape=(op.rows, op.rows))
    # Same number of iterations on both sides: the iterates agree up to rounding (GPU tree
    # reductions vs sequential sums). Mid-run iterates of this rank-deficient system are
    # sensitive -- a 1e-16 relative change of b alone moves the oracle's own iteration-15 field
    # by ~1e-8 on the torus before it settles again -- so the tight check is at 5 iterations;
    # an algorithmic difference would show at O(1) there.
    x_ref, _ = oracle.cgls(rp, col, val, b, 1e-300, 5, 0)
    x_gpu, r_gpu = op.solve(b, tol=1e-300, max_iters=5)
    assert r_gpu["iterations"] == 5
    assert np.linalg.norm(x_gpu - x_ref) <= 1e-10 * np.linalg.norm(x_ref)
    assert np.linalg.norm(A @ (x_gpu - x_ref)) <= 1e-10 * np.linalg.norm(b)
    # The GPU solve itself is deterministic: fixed-order reductions, bit-identical reruns.
    x_again, _ = op.solve(b, tol=1e-300, max_iters=5)
    assert np.array_equal(x_again, x_gpu)
    # Converged runs meet the same stopping test (possibly one iteration apart at the
    # threshold): their fitted fields differ by at most the two residuals.
    for tol, stop in [(1e-10, 0), (1e-6, 1)]:
        x_ref, r_ref = oracle.cgls(rp, col, val, b, tol, 1000, stop)
        x_gpu, r_gpu = op.solve(b, tol=tol, max_iters=1000, stop_rule=stop)
        assert r_gpu["converged"] and r_ref["converged"]
        assert abs(r_gpu["iterations"] - r_ref["iterations"]) <= 1
        bound = r_gpu["rel_residual"] + r_ref["rel_residual"] + 1e-11
        assert np.linalg.norm(A @ (x_gpu - x_ref)) <= bound * np.linalg.norm(b)
        rel = np.linalg.norm(A @ x_gpu - b) / np.linalg.norm(b)
        assert abs(rel - r_gpu["rel_residual"]) <= 1e-3 * rel + 1e-15
        if stop == 1:
            assert rel <= tol


@pytest.mark.gpu
def test_lscg_eigen_defaults_and_edge_cases(ctx):
    from its_b200 import Operator
    V, F, ref, gpu = _setup(ctx, "small", {}, 16)
    pos, _ = ref.vertices()
    b = oracle.signed_distance(pos, V, F)
    op = Operator(gpu)
    rp, col, val = ref.assemble()
    x_ref, r_ref = oracle.cgls(rp, col, val, b, 2.220446049250313e-16, 2 * op.rows, 0)
    x_gpu, r_gpu = op.solve(b)  # Eigen defaults: tol = eps, max 2n
    assert r_gpu["converged"] == r_ref["converged"]
    assert abs(r_gpu["iterations"] - r_ref["iterations"]) <= 0.1 * r_ref["iterations"] + 2
    A = sp.csr_matrix((val, col, rp), shape=(op.rows, op.rows))
    assert np.linalg.norm(A @ (x_gpu - x_ref)) <= 1e-12 * np.linalg.norm(b)
    # zero right-hand side: x = 0, zero iterations (Eigen's early exit)
    x0, r0 = op.solve(np.zeros(op.rows))
    assert r0["iterations"] == 0 and not np.any(x0)
    # warm start from the solution converges at once
    x1, r1 = op.solve(b, tol=1e-10, x0=x_gpu)
    assert r1["iterations"] <= 1
    # iteration cap is honoured and reported as not converged
    x2, r2 = op.solve(b, tol=1e-14, max_iters=3)
    assert r2["iterations"] == 3 and not r2["converged"]


@pytest.mark.gpu
def test_mixed_precision_reaches_tolerance(ctx):
    from its_b200 import OP_FP32_VALUES, PREC_MIXED, STOP_RESIDUAL, Operator
    V, F, ref, gpu = _setup(ctx, "c0", {}, 32)
    pos, _ = ref.vertices()
    b = oracle.signed_distance(pos, V, F)
    op = Operator(gpu, mode=OP_FP32_VALUES)
    x64, r64 = op.solve(b, tol=1e-6, stop_rule=STOP_RESIDUAL)
    xm, rm = op.solve(b, tol=1e-6, stop_rule=STOP_RESIDUAL, precision=PREC_MIXED, ir_steps=3, inner_tol=1e-3)
    assert rm["converged"] and rm["rel_residual"] <= 1e-6
    rp, col, val = op.csr()
    A = sp.csr_matrix((val, col, rp), shape=(op.rows, op.rows))
    assert np.linalg.norm(A @ xm - b) / np.linalg.norm(b) <= 1e-6
    # the field (A x) agrees with the FP64 solve to the residual level
    assert np.abs(A @ xm - A @ x64).max() <= 4e-6 * np.abs(b).max()


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,res", FIT_CASES[:2], ids=[f"{c[0]}-{c[2]}" for c in FIT_CASES[:2]])
def test_shell_samples_same_point_set(ctx, name, kw, res):
    V, F, ref, gpu = _setup(ctx, name, kw, res)
    pts_ref, ne_ref = ref.intersections()
    pts_gpu, ne_gpu = gpu.shell_samples(V, F)
    assert ne_gpu == ne_ref
    key = lambda P: P[np.lexsort((P[:, 2], P[:, 1], P[:, 0]))]  # noqa: E731
    assert np.array_equal(key(pts_gpu[:ne_gpu]), key(pts_ref[:ne_ref]))
    assert np.array_equal(key(pts_gpu[ne_gpu:]), key(pts_ref[ne_ref:]))


@pytest.mark.gpu
def test_batched_solve_matches_single_solves(ctx):
    from its_b200 import Operator, Svo
    from its_b200.api import solve_batch
    cases = [("small", {}, 16), ("c0", {}, 32), ("torus", dict(R=0.7, r=0.25, rings=48, segs=24), 32),
             ("superquadric", dict(e1=0.4, e2=2.5, subdiv=4), 16)]
    ops, bs = [], []
    for name, kw, res in cases:
        V, F, o, w = prepared_mesh(name, **kw)
        svo = Svo(ctx, V, F, res, o, w)
        pos, _ = svo.vertices()
        bs.append(ctx.signed_distance(pos, V, F))
        ops.append(Operator(svo))
    for tol, stop in [(1e-10, 0), (1e-6, 1)]:
        xs, reps = solve_batch(ops, bs, tol=tol, max_iters=1000, stop_rule=stop)
        for op, b, x, r in zip(ops, bs, xs, reps):
            xs1, r1 = op.solve(b, tol=tol, max_iters=1000, stop_rule=stop)
            # the same per-mesh algorithm; only the chunking of the dot products differs
            assert r["converged"] and abs(r["iterations"] - r1["iterations"]) <= 1
            rp, col, val = op.csr()
            A = sp.csr_matrix((val, col, rp), shape=(op.rows, op.rows))
            assert np.linalg.norm(A @ (x - xs1)) <= (r["rel_residual"] + r1["rel_residual"] + 1e-11) * np.linalg.norm(b)
            assert abs(np.linalg.norm(A @ x - b) / np.linalg.norm(b) - r["rel_residual"]) <= 1e-3 * r["rel_residual"] + 1e-15
    # a zero right-hand side in the batch finishes at once with x = 0
    xs, reps = solve_batch(ops[:2], [bs[0], np.zeros(ops[1].rows)], tol=1e-8)
    assert reps[1]["iterations"] == 0 and not np.any(xs[1]) and reps[0]["converged"]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,res", FIT_CASES, ids=[f"{c[0]}-{c[2]}" for c in FIT_CASES])
def test_exact_start_matches_oracle(ctx, name, kw, res):
    from its_b200 import Operator
    V, F, ref, gpu = _setup(ctx, name, kw, res)
    pos, _ = ref.vertices()
    b = oracle.signed_distance(pos, V, F)
    op = Operator(gpu)
    rp, col, val = ref.assemble()
    A = sp.csr_matrix((val, col, rp), shape=(op.rows, op.rows))
    # zero shares: an exact solution; the GPU generates each row's parent-cell hats from the
    # octree and sums them in column order like the oracle, so the two are bit-identical
    lam_ref = ref.exact_start(b)
    lam = gpu.exact_start(b)
    assert np.array_equal(lam, lam_ref)
    assert np.linalg.norm(A @ lam - b) <= 1e-14 * np.linalg.norm(b)
    # the matrix-free residual agrees with the assembled operator's, up to the rounding of the
    # row sums (summed in another order: each entry of A lam within k eps (|A| |lam|)_i, k <= 64)
    rel = np.linalg.norm(A @ lam - b) / np.linalg.norm(b)
    sum_err = 64 * np.finfo(float).eps * np.linalg.norm(abs(A) @ np.abs(lam)) / np.linalg.norm(b)
    assert abs(gpu.residual(b, lam) - rel) <= 1e-3 * rel + sum_err
    # and away from a solution (the level recursion evaluates the same A lambda)
    x_r = np.random.default_rng(3).standard_normal(op.rows)
    rel_r = np.linalg.norm(A @ x_r - b) / np.linalg.norm(b)
    assert abs(gpu.residual(b, x_r) - rel_r) <= 1e-12 * rel_r
    # CGLS started there stops at its residual test
    x, rep = op.solve(b, tol=1e-6, stop_rule=1, x0=lam)
    assert rep["iterations"] == 0 and rep["converged"] and rep["rel_residual"] <= 1e-14
    # the shares fix the null-space component: the min-norm shares give back the (zero-start)
    # CGLS solution, and every exact solution has the same field at the shell samples
    x_mn, _ = oracle.cgls(rp, col, val, b, 1e-14, 20000, 1)
    lam_mn = gpu.exact_start(b, shares=x_mn)
    assert np.array_equal(lam_mn, ref.exact_start(b, shares=x_mn))
    assert np.abs(lam_mn - x_mn).max() <= 1e-12 * np.abs(x_mn).max()
    P = np.vstack([V, ref.intersections()[0]])
    f0, _ = ref.eval_points(lam, P)
    f1, _ = ref.eval_points(x_mn, P)
    assert np.abs(f0 - f1).max() <= 1e-12 * np.abs(b).max()


@pytest.mark.gpu
def test_exact_start_batch_matches_single(ctx):
    from its_b200 import Svo
    from its_b200.api import exact_start_batch, fit_residual_batch
    svos, bs = [], []
    for name, kw, res in FIT_CASES + [("superquadric", dict(e1=0.4, e2=2.5, subdiv=4), 64)]:
        V, F, o, w = prepared_mesh(name, **kw)
        svo = Svo(ctx, V, F, res, o, w)
        bs.append(ctx.signed_distance(svo.vertices()[0], V, F))
        svos.append(svo)
    rng = np.random.default_rng(5)
    shares = [None, rng.standard_normal(svos[1].num_verts) * 1e-3, None, None]
    outs = exact_start_batch(svos, bs, shares)
    rels = fit_residual_batch(svos, bs, outs)
    for svo, b, s, x, r in zip(svos, bs, shares, outs, rels):
        assert np.array_equal(x, svo.exact_start(b, shares=s))
        assert r == svo.residual(b, x) and r <= 1e-14
    # more octrees than a launch carries inline (16): the tables go through device memory
    many = [(svos[k % 4], bs[k % 4], shares[k % 4]) for k in range(19)]
    outs = exact_start_batch([m[0] for m in many], [m[1] for m in many], [m[2] for m in many])
    rels = fit_residual_batch([m[0] for m in many], [m[1] for m in many], outs)
    for (svo, b, s), x, r in zip(many, outs, rels):
        assert np.array_equal(x, svo.exact_start(b, shares=s))
        assert r == svo.residual(b, x)


@pytest.mark.gpu
def test_copy_to_device_small_and_staged(ctx):
    # its_copy_to_device: a small array by one copy, a large pageable one through the pinned
    # chunks filled by host threads (also the path of every large host input)
    rng = np.random.default_rng(3)
    for n in (1000, 5_000_001, 9_000_001):  # 8 KB, 40 MB (below the staged size), 72 MB (pieces, odd tail)
        a = rng.standard_normal(n)
        assert np.array_equal(ctx.to_device(a).cpu().numpy(), a)
    f = rng.integers(0, 1 << 30, size=(6_000_000, 3)).astype(np.int32)
    assert np.array_equal(ctx.to_device(f).cpu().numpy(), f)
