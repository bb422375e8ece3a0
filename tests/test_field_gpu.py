"""Field-path parity: point evaluation, iso levels, dense lattice field and marching cubes.

Bars: point evaluation and the lattice field use the oracle's terms in the oracle's order
and are bit-exact; marching-cubes case indices are bit-exact for the same lattice field and
the triangle soup is identical (same lerp with explicit fma). The fit identity of the
reference (field at corner vertices = b, ThinShells.cpp:629-652) holds to the solve
tolerance.
"""
import numpy as np
import pytest

import oracle
from cascade_np import cascade_numpy as _cascade_numpy
from conftest import prepared_mesh


def _fit(ctx, name="c0", res=32, tol=1e-12):
    from its_b200 import Operator, Svo
    V, F, o, w = prepared_mesh(name)
    ref, gpu = oracle.Svo(V, F, res, o, w), Svo(ctx, V, F, res, o, w)
    pos, _ = ref.vertices()
    b = oracle.signed_distance(pos, V, F)
    lam, rep = Operator(gpu).solve(b, tol=tol, max_iters=2000)
    return V, F, o, w, ref, gpu, pos, b, lam


@pytest.fixture(scope="module")
def fitted(ctx):
    return _fit(ctx)


@pytest.mark.gpu
def test_eval_points_bit_exact_and_interpolates(fitted):
    V, F, o, w, ref, gpu, pos, b, lam = fitted
    samples = np.vstack([V, pos])
    f_gpu, m_gpu = gpu.eval_points(lam, samples)
    f_ref, m_ref = ref.eval_points(lam, samples)
    assert np.array_equal(m_gpu, m_ref)
    assert np.array_equal(f_gpu, f_ref)
    # interpolation identity at corner vertices that lie in a fine node
    fv = f_gpu[len(V):]
    inside = m_gpu[len(V):] == 0
    assert np.abs(fv[inside] - b[inside]).max() <= 1e-9


@pytest.mark.gpu
def test_shell_iso_values(fitted):
    V, F, o, w, ref, gpu, pos, b, lam = fitted
    pts, _ = gpu.shell_samples(V, F)
    samples = np.vstack([V, pts])
    lo, hi, miss = gpu.shell_iso_values(lam, samples)
    f_ref, m_ref = ref.eval_points(lam, samples)
    assert miss == int(m_ref.sum())
    assert lo == f_ref[m_ref == 0].min() and hi == f_ref[m_ref == 0].max()
    assert lo < 0 < hi


@pytest.mark.gpu
@pytest.mark.parametrize("R", [32, 64])
def test_grid_field_bit_exact_and_matches_brute_force(fitted, R):
    V, F, o, w, ref, gpu, pos, b, lam = fitted
    g_gpu = gpu.eval_grid(lam, o, w, R)
    g_ref = ref.eval_grid(lam, o, w, R)
    assert np.array_equal(g_gpu, g_ref)
    M = R + 1
    idx = np.random.default_rng(0).choice(M ** 3, 500, replace=False)
    xi, yj, zk = idx % M, (idx // M) % M, idx // (M * M)
    P = np.stack([o[0] + xi * (w[0] / R), o[1] + yj * (w[1] / R), o[2] + zk * (w[2] / R)], 1)
    brute = ref.eval_brute(lam, P)
    assert np.allclose(g_gpu[idx], brute, rtol=0, atol=1e-14)


@pytest.mark.gpu
def test_point_query_bit_exact(fitted):
    V, F, o, w, ref, gpu, pos, b, lam = fitted
    pts, _ = gpu.shell_samples(V, F)
    lo, hi, _ = gpu.shell_iso_values(lam, np.vstack([V, pts]))
    e = o + w
    rng = np.random.default_rng(5)
    P = np.vstack([o - w + 3 * w * rng.random((3000, 3)),          # includes points outside the range
                   V[:500] + rng.normal(0, 1e-3, (500, 3))])       # near the surface
    v_gpu, l_gpu = gpu.point_query(lam, P, o, e, lo, hi)
    v_ref, l_ref = ref.point_query(lam, P, o, e, lo, hi)
    assert np.array_equal(v_gpu, v_ref) and np.array_equal(l_gpu, l_ref)
    assert set(np.unique(l_gpu)) == {-1, 0, 1}
    inside = np.all((P >= o - w) & (P <= e + w), axis=1)
    brute = ref.eval_brute(lam, P[inside][:400])
    assert np.allclose(v_gpu[inside][:400], brute, rtol=0, atol=1e-14)
    assert np.all(v_gpu[~inside] == hi)


@pytest.mark.gpu
def test_welded_mc_mesh(ctx, fitted):
    V, F, o, w, ref, gpu, pos, b, lam = fitted
    R = 40
    field = gpu.eval_grid(lam, o, w, R)
    verts, tris = ctx.marching_cubes_mesh(field, R, o, w, 0.0)
    rv, rt = oracle.marching_cubes_mesh(field, R, o, w, 0.0)
    assert np.array_equal(verts, rv) and np.array_equal(tris, rt)
    # same surface as the soup: every soup vertex is a welded vertex (up to the lerp's end
    # point order), and the soup has 3 vertices per welded triangle
    _, soup, n = ctx.marching_cubes(field, R, o, w, 0.0)
    assert n == 3 * len(tris)
    assert np.abs(verts[tris.reshape(-1)] - soup).max() <= 1e-12
    # welded: edges are shared by two triangles (the classic table may leave a few open edges
    # at ambiguous faces, never more than two triangles on one edge)
    e = np.sort(np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]]), axis=1)
    _, counts = np.unique(e, axis=0, return_counts=True)
    assert counts.max() <= 2 and (counts == 2).mean() > 0.99


@pytest.mark.gpu
@pytest.mark.parametrize("R", [16, 48])
def test_marching_cubes_bit_exact(ctx, fitted, R):
    V, F, o, w, ref, gpu, pos, b, lam = fitted
    field = gpu.eval_grid(lam, o, w, R)
    f, miss = ref.eval_points(lam, V)
    for iso in (f.min(), 0.0, f.max()):
        cube_g, tri_g, n_g = ctx.marching_cubes(field, R, o, w, iso)
        cube_r, tri_r, n_r = oracle.marching_cubes(field, R, o, w, iso)
        assert n_g == n_r and n_g > 0
        assert np.array_equal(cube_g, cube_r)
        assert np.array_equal(tri_g, tri_r)


@pytest.mark.gpu
def test_marching_cubes_bit_exact_tiled_block_sum_scan(ctx, fitted):
    # At R = 260 the classify pass leaves 8,583 block sums (2,048 voxels each): above the 8,192
    # that one block scans, so the spine runs in tiles of 2,048 with a partial last tile; the
    # cases and the soup stay the oracle's.
    V, F, o, w, ref, gpu, pos, b, lam = fitted
    R = 260
    field = gpu.eval_grid(lam, o, w, R)
    cube_g, tri_g, n_g = ctx.marching_cubes(field, R, o, w, 0.0)
    cube_r, tri_r, n_r = oracle.marching_cubes(field, R, o, w, 0.0)
    assert n_g == n_r and n_g > 0
    assert np.array_equal(cube_g, cube_r)
    assert np.array_equal(tri_g, tri_r)


@pytest.mark.gpu
def test_fast_division_is_correctly_rounded(ctx):
    # The field kernels divide by the cell width through RN(1/w) and two FMAs (Markstein);
    # the quotients must equal the GPU's correctly rounded division bit for bit.
    import ctypes as C
    from its_b200 import lib
    rng = np.random.default_rng(0)
    n = 1 << 22
    a = rng.standard_normal(n) * np.exp(rng.uniform(-30, 30, n))
    b = rng.standard_normal(n) * np.exp(rng.uniform(-30, 30, n))
    # the kernels' own operands: offsets within two cells of widths w0 * 2^d
    w = (1.18 / 256) * 2.0 ** rng.integers(0, 10, n)
    a2 = rng.uniform(-2, 2, n) * w
    # and exact multiples / neighbours of them, the ties of a floor
    k = rng.integers(-600, 600, n).astype(np.float64)
    a3 = np.nextafter(k * w, k * w + rng.choice([-1.0, 1.0], n))
    for x, y in ((a, b), (a2, w), (a3, w), (k * w, w)):
        miss = C.c_int64(-1)
        ctx.check(lib().its_check_division(ctx.h, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p), n,
                                           C.byref(miss)), "its_check_division")
        assert miss.value == 0


@pytest.mark.gpu
def test_fp32_field_and_marching_cubes(ctx):
    # Precision mode: the FP32 field agrees with the FP64 one to FP32 rounding, and FP32
    # marching cubes gives the same case indices outside the band where FP32 rounding can
    # move a corner across the iso level.
    import ctypes as C
    from its_b200 import Operator, Svo, lib
    V, F, o, w = prepared_mesh("c0")
    svo = Svo(ctx, V, F, 32, o, w)
    b = ctx.signed_distance(svo.vertices()[0], V, F)
    lam, _ = Operator(svo).solve(b, tol=1e-10, max_iters=1000)
    R = 96
    f64 = svo.eval_grid(lam, o, w, R)
    f32 = svo.eval_grid_f32(lam, o, w, R)
    scale = np.abs(f64).max()
    err = np.abs(f32.astype(np.float64) - f64)
    assert err.max() <= 2e-6 * scale, err.max() / scale
    iso = float(np.median(b[np.abs(b) < 0.05]))
    cubes = []
    for fld, fn in ((f64, lib().its_marching_cubes), (f32, lib().its_marching_cubes_f32)):
        cube = np.zeros(R ** 3, np.uint8)
        n = C.c_int64(0)
        ctx.check(fn(ctx.h, fld.ctypes.data_as(C.c_void_p), R, o.ctypes.data_as(C.c_void_p),
                     w.ctypes.data_as(C.c_void_p), iso, cube.ctypes.data_as(C.c_void_p), None, 0, C.byref(n)), "mc")
        cubes.append(cube)
    diff = np.nonzero(cubes[0] != cubes[1])[0]
    M = R + 1
    g = f64.reshape(M, M, M)  # [z][y][x]
    for v in diff:
        x, y, z = v % R, (v // R) % R, v // (R * R)
        corners = g[z:z + 2, y:y + 2, x:x + 2]
        assert np.abs(corners - iso).min() <= 4e-6 * scale
    assert len(diff) <= 1e-3 * R ** 3


@pytest.mark.gpu
def test_autotuner_changes_speed_not_bits(tmp_path):
    # Tuned launches (brick shape of the dense field, marching-cubes tile) compute the same
    # bits as the defaults; the choices are recorded and persist through the cache file.
    from its_b200 import Context, Operator, Svo
    V, F, o, w = prepared_mesh("c0")
    outs = {}
    cache = str(tmp_path / "tune.txt")
    for mode in (0, 1, 2):
        ctx = Context(0)
        if mode:
            ctx.set_autotune(True, cache)
        svo = Svo(ctx, V, F, 32, o, w)
        b = ctx.signed_distance(svo.vertices()[0], V, F)
        lam = svo.exact_start(b)
        field = svo.eval_grid(lam, o, w, 80)
        cube, tri, n = ctx.marching_cubes(field, 80, o, w, float(np.median(b)))
        field32 = svo.eval_grid_f32(lam, o, w, 80)
        outs[mode] = (field, cube, tri, ctx.autotune_choices(), field32)
        ctx.close()
    for mode in (1, 2):
        assert np.array_equal(outs[mode][0], outs[0][0]) and np.array_equal(outs[mode][4], outs[0][4])
        assert np.array_equal(outs[mode][1], outs[0][1]) and np.array_equal(outs[mode][2], outs[0][2])
    choices = outs[1][3]
    assert any(k.startswith("eval_grid/f64") for k in choices) and any(k.startswith("marching_cubes/f64") for k in choices)
    assert outs[2][3] == choices  # read back from the cache file


@pytest.mark.gpu
def test_every_tuned_candidate_computes_the_same_bits(tmp_path):
    # Each launch shape the autotuner may pick -- the four brick shapes and the two separable
    # depths of the FP64 field, the two separable depths of the FP32 field, the three
    # marching-cubes tiles -- forced through the cache file in turn, gives the defaults' bits.
    from its_b200 import Context, Svo
    V, F, o, w = prepared_mesh("c0")
    R = 80

    def run(cache=None):
        ctx = Context(0)
        if cache:
            ctx.set_autotune(True, cache)
        svo = Svo(ctx, V, F, 32, o, w)
        b = ctx.signed_distance(svo.vertices()[0], V, F)
        lam = svo.exact_start(b)
        field = svo.eval_grid(lam, o, w, R)
        field32 = svo.eval_grid_f32(lam, o, w, R)
        cube, tri, n = ctx.marching_cubes(field, R, o, w, float(np.median(b)))
        out = (field, field32, cube, tri, svo.depth, ctx.autotune_choices())
        ctx.close()
        return out

    ref = run()
    depth = ref[4]
    for k in range(6):
        cache = str(tmp_path / ("tune%d.txt" % k))
        with open(cache, "w") as f:
            f.write("eval_grid/f64/grid=%d/octree=32/depth=%d %d\n" % (R, depth, k))
            f.write("eval_grid/f32/grid=%d/octree=32/depth=%d %d\n" % (R, depth, k % 2))
            f.write("marching_cubes/f64/res=%d/cases %d\n" % (R, k % 3))
            f.write("marching_cubes/f64/res=%d/soup %d\n" % (R, k % 3))
        got = run(cache)
        assert got[5]["eval_grid/f64/grid=%d/octree=32/depth=%d" % (R, depth)] == k
        assert got[5]["eval_grid/f32/grid=%d/octree=32/depth=%d" % (R, depth)] == k % 2
        assert got[5]["marching_cubes/f64/res=%d/cases" % R] == got[5]["marching_cubes/f64/res=%d/soup" % R] == k % 3
        assert np.array_equal(got[0], ref[0]), "FP64 field, candidate %d" % k
        assert np.array_equal(got[1], ref[1]), "FP32 field, candidate %d" % (k % 2)
        assert np.array_equal(got[2], ref[2]) and np.array_equal(got[3], ref[3]), "marching cubes, tile %d" % (k % 3)


@pytest.mark.gpu
def test_point_value_gradient_matches_oracle(ctx):
    from its_b200 import Operator, Svo, uniform_bbox
    V, F, o, w = prepared_mesh("c0")
    ref = oracle.Svo(V, F, 32, o, w)
    svo = Svo(ctx, V, F, 32, o, w)
    b = oracle.signed_distance(ref.vertices()[0], V, F)
    lam, _ = Operator(svo).solve(b, tol=1e-10, max_iters=1000)
    bo, be, _ = uniform_bbox(V)
    rng = np.random.default_rng(4)
    P = np.vstack([V + rng.normal(0, 0.01, V.shape), bo + (be - bo) * rng.uniform(-0.3, 1.3, (2000, 3))])
    before = V[rng.integers(0, len(V), len(P))]
    for bf in (None, before):
        v, g, miss = svo.point_gradient(lam, P, bo, be, bf)
        v_r, g_r, miss_r = ref.point_gradient(lam, P, bo, be, bf)
        assert np.array_equal(miss, miss_r) and np.array_equal(v, v_r) and np.array_equal(g, g_r)
    # the gradient is the field's derivative: central differences inside fine cells
    h = 1e-7
    inside = np.nonzero(miss == 0)[0][:200]
    for a in range(3):
        e = np.zeros(3)
        e[a] = h
        fp, _, mp = svo.point_gradient(lam, P[inside] + e, bo, be)
        fm, _, mm = svo.point_gradient(lam, P[inside] - e, bo, be)
        ok = (mp == 0) & (mm == 0)
        fd = (fp - fm) / (2 * h)
        assert np.median(np.abs(fd[ok] - g[inside][ok, a])) <= 1e-5 * np.abs(g[inside]).max()


@pytest.mark.gpu
@pytest.mark.parametrize("f", [1, 2, 4])
def test_grid_field_by_prolongation(fitted, f):
    # on the octree's own lattice (res * f): the cascade equals its numpy restatement to
    # rounding, and the point-by-point field to the geometry's single-precision offsets (corner
    # positions and a float-padded box a few 1e-9 off the lattice: ~1e-8 of max |field|); FP32
    # within FP32 rounding; a lattice off the octree's falls back to the exact evaluator
    V, F, o, w, ref, gpu, pos, b, lam = fitted
    res = 32
    R = res * f
    M = R + 1
    exact = gpu.eval_grid(lam, o, w, R)
    fast = gpu.eval_grid_fast(lam, o, w, R)
    scale = np.abs(exact).max()
    assert np.abs(fast - exact).max() <= 1e-6 * scale
    unit = np.full(3, np.asarray(w, float)[0] / res)  # the octree sizes its cells by its first axis
    cas = _cascade_numpy(pos, lam, gpu.depth_counts()[1], np.asarray(o, float), unit, res, f)
    assert np.abs(fast.reshape(M, M, M).transpose(2, 1, 0) - cas).max() <= 1e-13 * scale
    f32 = gpu.eval_grid_fast(lam, o, w, R, fp32=True)
    assert np.abs(f32.astype(np.float64) - exact).max() <= 1e-5 * scale
    shifted = np.asarray(o, float) + 0.25 * unit
    assert np.array_equal(gpu.eval_grid_fast(lam, shifted, w, R), gpu.eval_grid(lam, shifted, w, R))


@pytest.mark.gpu
def test_marching_cubes_row_tiles_bit_exact(ctx, fitted):
    # grids whose side is a multiple of 256 classify with row tiles (coalesced loads, lanes on
    # interleaved voxels): the same case bytes and triangles as the oracle, FP64 and FP32
    import ctypes as C
    from its_b200 import lib
    V, F, o, w, ref, gpu, pos, b, lam = fitted
    R = 256
    field = gpu.eval_grid_fast(lam, o, w, R)
    iso = float(np.median(b[np.abs(b) < 0.05]))
    cube_g, tri_g, n_g = ctx.marching_cubes(field, R, o, w, iso)
    cube_r, tri_r, n_r = oracle.marching_cubes(field, R, o, w, iso)
    assert n_g == n_r and n_g > 0
    assert np.array_equal(cube_g, cube_r)
    assert np.array_equal(tri_g, tri_r)
    f32 = field.astype(np.float32)
    cube = np.zeros(R ** 3, np.uint8)
    n = C.c_int64(0)
    o_, w_ = np.ascontiguousarray(o, np.float64), np.ascontiguousarray(w, np.float64)
    ctx.check(lib().its_marching_cubes_f32(ctx.h, f32.ctypes.data_as(C.c_void_p), R, o_.ctypes.data_as(C.c_void_p),
                                           w_.ctypes.data_as(C.c_void_p), iso, cube.ctypes.data_as(C.c_void_p), None, 0,
                                           C.byref(n)), "mc f32")
    cube_r32, _, n_r32 = oracle.marching_cubes(f32.astype(np.float64), R, o, w, iso)
    assert np.array_equal(cube, cube_r32) and n.value == n_r32


@pytest.mark.gpu
@pytest.mark.parametrize("fast", [False, True])
def test_grid_mc_driver_matches_field_then_marching_cubes(ctx, fitted, fast):
    # its_eval_grid_mc (the mcVisualization driver, field kept on the device) gives exactly the
    # soups of its_eval_grid / its_eval_grid_fast followed by its_marching_cubes per level
    V, F, o, w, ref, gpu, pos, b, lam = fitted
    R = 64  # 2 x the octree's res: the prolongation lattice
    field = gpu.eval_grid_fast(lam, o, w, R) if fast else gpu.eval_grid(lam, o, w, R)
    isos = [float(np.quantile(field, 0.4)), float(np.quantile(field, 0.6)), 0.0]
    soups = gpu.grid_mc(lam, o, w, R, isos, fast=fast)
    counts = gpu.grid_mc(lam, o, w, R, isos, fast=fast, triangles=False)
    for iso, soup, cnt in zip(isos, soups, counts):
        _, tri, n = ctx.marching_cubes(field, R, o, w, iso)
        assert n == cnt == soup.shape[0] and n > 0
        assert np.array_equal(soup, tri)
