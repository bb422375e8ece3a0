"""The cubic tensor-product B-spline basis and the offset shell samples (no counterpart in the
reference, whose basis is the degree-1 hat of BSpline.hpp:4-22): libits against the oracle's
restatement (oracle/orc_cubic.cpp).

Bars: offset samples, the assembled cubic system (corner-vertex rows and offset-sample rows)
and the field at points and on lattices are bit-exact with the oracle (same terms in the same
order); the fit (FP64 LSCG) agrees with the oracle's CGLS after the same number of iterations
to 1e-6 relative in the coefficients and 1e-9 in the relative residual; marching-cubes case indices of the GPU's fitted field are bit-exact with the
oracle's marching cubes on the oracle's field of the same coefficients.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from conftest import prepared_mesh


def _setup(ctx, name="c0", res=32, kw=None):
    from its_b200 import Svo
    V, F, o, w = prepared_mesh(name, **(kw or {}))
    eps = 0.01 * float(np.linalg.norm(V.max(0) - V.min(0)))
    return V, F, o, w, eps, oracle.Svo(V, F, res, o, w), Svo(ctx, V, F, res, o, w)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c0", "small"])
def test_offset_samples_bit_exact(ctx, name):
    V, F, o, w = prepared_mesh(name)
    eps = 0.01 * float(np.linalg.norm(V.max(0) - V.min(0)))
    P, T = ctx.offset_samples(V, F, eps)
    Pr, Tr = oracle.offset_samples(V, F, eps)
    assert np.array_equal(P, Pr) and np.array_equal(T, Tr)
    nv = len(V)
    d = P[:nv] - V
    assert np.allclose(np.linalg.norm(d, axis=1), eps, rtol=1e-12)  # one eps along a unit normal
    assert np.array_equal(P[nv:] - V, -(P[:nv] - V)) or np.allclose(P[nv:] - V, -d, atol=1e-15)


@pytest.mark.gpu
@pytest.mark.parametrize("name,res,with_samples", [("c0", 32, True), ("small", 16, False), ("c0", 16, True)])
def test_cubic_operator_bit_exact(ctx, name, res, with_samples):
    from its_b200 import Operator
    V, F, o, w, eps, ref, gpu = _setup(ctx, name, res)
    P = ctx.offset_samples(V, F, eps)[0] if with_samples else None
    op = Operator(gpu, degree=3, samples=P)
    rp, col, val = op.csr()
    orp, ocol, oval = ref.cubic_assemble(P)
    assert op.rows == len(orp) - 1 == gpu.num_verts + (0 if P is None else len(P))
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol) and np.array_equal(val, oval)
    op.close()


@pytest.mark.gpu
def test_cubic_field_bit_exact(ctx):
    V, F, o, w, eps, ref, gpu = _setup(ctx)
    rng = np.random.default_rng(7)
    lam = rng.standard_normal(gpu.num_verts)
    P = np.vstack([V, rng.uniform(o, o + w, (2000, 3))])
    assert np.array_equal(gpu.eval_points_cubic(lam, P), ref.cubic_eval(lam, P))
    for R in (32, 48):
        assert np.array_equal(gpu.eval_grid_cubic(lam, o, w, R), ref.cubic_eval_grid(lam, o, w, R))
    # the rows of the assembled system are the field at their points (the SpMV splits long rows
    # over lanes, so its sums run in another order: 1e-13 relative)
    from its_b200 import Operator
    Ps = ctx.offset_samples(V, F, eps)[0]
    op = Operator(gpu, degree=3, samples=Ps)
    x = np.concatenate([lam, np.zeros(len(Ps))])
    Ax = op.apply(x)
    f = gpu.eval_points_cubic(lam, Ps)
    assert np.abs(Ax[gpu.num_verts:] - f).max() <= 1e-13 * np.abs(f).max()
    op.close()


@pytest.mark.gpu
def test_cubic_fit_with_offset_samples_c0(ctx):
    """c0 of the workload list: cubic basis, corner vertices (signed distance) and offset shell
    samples (+-0.01 diag), FP64 LSCG; marching cubes at 128^3 at the shell iso levels."""
    from its_b200 import Operator
    V, F, o, w, eps, ref, gpu = _setup(ctx)
    Ps, Ts = ctx.offset_samples(V, F, eps)
    pos, _ = gpu.vertices()
    b = np.concatenate([ctx.signed_distance(pos, V, F), Ts])
    op = Operator(gpu, degree=3, samples=Ps)
    K = 40
    lam, rep = op.solve(b, tol=1e-10, max_iters=K)
    rp, col, val = ref.cubic_assemble(Ps)
    lam_ref, rep_ref = oracle.cgls(rp, col, val, b, 1e-10, K, 0)
    assert rep["iterations"] == rep_ref["iterations"] == K
    # the same CGLS; the SpMV's summation order differs, and the redundant cubic system
    # amplifies that rounding over the iterations: 1e-6 relative in lambda, residuals to 1e-9
    assert np.linalg.norm(lam - lam_ref) <= 1e-6 * np.linalg.norm(lam_ref)
    assert abs(rep["rel_residual"] - rep_ref["rel_residual"]) <= 1e-9
    assert np.all(lam[gpu.num_verts:] == 0.0)
    A = sp.csr_matrix((val, col, rp), shape=(len(rp) - 1,) * 2)
    rel = np.linalg.norm(b - A @ lam) / np.linalg.norm(b)
    assert abs(rel - rep["rel_residual"]) <= 1e-9 and rel < 0.05
    n = gpu.num_verts
    f_off = gpu.eval_points_cubic(lam[:n], Ps)
    assert np.abs(f_off - Ts).max() <= 0.5 * eps  # the fit separates the two offset shells
    samples = np.vstack([V, gpu.shell_samples(V, F)[0]])
    fs = gpu.eval_points_cubic(lam[:n], samples)
    R = 128
    field = gpu.eval_grid_cubic(lam[:n], o, w, R)
    field_ref = ref.cubic_eval_grid(lam[:n], o, w, R)
    assert np.array_equal(field, field_ref)
    for iso in (fs.min(), fs.max()):
        cube, _, nverts = ctx.marching_cubes(field, R, o, w, iso, triangles=False)
        cube_ref, _, n_ref = oracle.marching_cubes(field_ref, R, o, w, iso, with_triangles=False)
        assert nverts == n_ref > 0 and np.array_equal(cube, cube_ref)
    op.close()


@pytest.mark.gpu
def test_cubic_rejects_bad_options(ctx):
    import ctypes as C
    from its_b200 import lib
    from its_b200._lib import BasisOpts
    V, F, o, w, eps, ref, gpu = _setup(ctx, "small", 8)
    h = C.c_void_p()
    for opts in (BasisOpts(2, None, 0), BasisOpts(1, None, 5), BasisOpts(3, None, 4)):
        assert lib().its_operator_build_ex(gpu.h, 0, C.byref(opts), C.byref(h)) == 1
