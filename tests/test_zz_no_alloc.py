"""its_marching_cubes_noalloc: marching cubes for callers that cannot let the library allocate
device memory (an application that keeps the GPU's memory in its own fixed budget, or a frame
loop that cudaMalloc's implicit device synchronisation would stall). Its scan scratch is a fixed
file-scope device array, so it must return exactly what the allocating its_marching_cubes
returns, on consecutive calls that reuse that array, up to the largest size the array holds
(res 256, where the spine fills all 8,192 block-sum words). This file is collected last on
purpose."""
import ctypes as C

import numpy as np
import pytest

from conftest import prepared_mesh


def _fitted_field(ctx, R):
    import oracle
    from its_b200 import Operator, Svo
    V, F, o, w = prepared_mesh("c0")
    svo = Svo(ctx, V, F, 32, o, w)
    pos, _ = svo.vertices()
    b = oracle.signed_distance(pos, V, F)
    lam, _ = Operator(svo).solve(b, tol=1e-8, max_iters=1000)
    return svo.eval_grid(lam, o, w, R), o, w


def _analytic_field(R):
    """A wavy sphere's implicit function on the (R+1)^3 lattice of the unit box, x fastest."""
    t = np.linspace(0.0, 1.0, R + 1)
    z, y, x = np.meshgrid(t, t, t, indexing="ij")
    r = np.sqrt((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2)
    return (r - 0.3 - 0.03 * np.sin(9 * x) * np.cos(7 * y)).reshape(-1), np.zeros(3), np.ones(3)


def _declare(L):
    L.its_marching_cubes_noalloc.restype = C.c_int
    L.its_marching_cubes_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                                             C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _check_case(L, ctx, field, R, o, w, iso):
    """Both entry points on one field; the allocation-free one twice in a row (tolerance: bit-exact,
    as the allocating path)."""
    import torch
    po, pw = o.ctypes.data_as(C.c_void_p), w.ctypes.data_as(C.c_void_p)
    n_ref = C.c_int64(0)
    ctx.check(L.its_marching_cubes(ctx.h, _ptr(field), R, po, pw, iso, None, None, 0, C.byref(n_ref)), "mc")
    assert n_ref.value > 0
    cube_ref = torch.zeros(R ** 3, dtype=torch.uint8, device="cuda")
    tri_ref = torch.zeros(3 * n_ref.value, dtype=torch.float64, device="cuda")
    ctx.check(L.its_marching_cubes(ctx.h, _ptr(field), R, po, pw, iso, _ptr(cube_ref), _ptr(tri_ref),
                                   n_ref.value, C.byref(n_ref)), "mc")
    for _ in range(2):  # two calls in a row through the shared scratch array
        n = C.c_int64(-1)
        cube = torch.full((R ** 3,), 255, dtype=torch.uint8, device="cuda")
        tri = torch.full((3 * n_ref.value,), np.nan, dtype=torch.float64, device="cuda")
        ctx.check(L.its_marching_cubes_noalloc(ctx.h, _ptr(field), R, po, pw, iso, _ptr(cube), _ptr(tri),
                                               n_ref.value, C.byref(n)), "mc noalloc")
        assert n.value == n_ref.value
        assert torch.equal(cube, cube_ref)
        assert torch.equal(tri, tri_ref)
    # counts only: both outputs NULL, and cube indices without triangles
    n = C.c_int64(-1)
    ctx.check(L.its_marching_cubes_noalloc(ctx.h, _ptr(field), R, po, pw, iso, None, None, 0, C.byref(n)), "count")
    assert n.value == n_ref.value
    cube = torch.zeros(R ** 3, dtype=torch.uint8, device="cuda")
    ctx.check(L.its_marching_cubes_noalloc(ctx.h, _ptr(field), R, po, pw, iso, _ptr(cube), None, 0, C.byref(n)),
              "cubes only")
    assert n.value == n_ref.value and torch.equal(cube, cube_ref)
    # a buffer for half the soup: the first half is written, num_verts is still the full total
    half = n_ref.value // 2
    tri = torch.full((3 * n_ref.value,), np.nan, dtype=torch.float64, device="cuda")
    ctx.check(L.its_marching_cubes_noalloc(ctx.h, _ptr(field), R, po, pw, iso, None, _ptr(tri), half, C.byref(n)),
              "half capacity")
    assert n.value == n_ref.value
    assert torch.equal(tri[:3 * half], tri_ref[:3 * half])
    assert bool(torch.isnan(tri[3 * half:]).all())


@pytest.mark.gpu
def test_noalloc_marching_cubes_matches_allocating_entry_point():
    import torch
    from its_b200 import Context, lib
    L = lib()
    _declare(L)
    ctx = Context(0)
    try:
        R = 96
        field_h, o, w = _fitted_field(ctx, R)
        field = torch.from_numpy(field_h).cuda()
        for iso in (float(np.quantile(field_h, 0.3)), 0.0):
            _check_case(L, ctx, field, R, o, w, iso)
        # the largest size the fixed scratch holds: res 256 fills every block-sum word
        R = 256
        field_h, o, w = _analytic_field(R)
        field = torch.from_numpy(field_h).cuda()
        _check_case(L, ctx, field, R, o, w, 0.0)
        # limits: sizes beyond the fixed scratch and host buffers are refused
        po, pw = o.ctypes.data_as(C.c_void_p), w.ctypes.data_as(C.c_void_p)
        n = C.c_int64(0)
        big = torch.zeros(1, dtype=torch.float64, device="cuda")
        assert L.its_marching_cubes_noalloc(ctx.h, _ptr(big), 257, po, pw, 0.0, None, None, 0, C.byref(n)) == 1
        assert L.its_marching_cubes_noalloc(ctx.h, field_h.ctypes.data_as(C.c_void_p), R, po, pw, 0.0, None, None, 0,
                                            C.byref(n)) == 1
    finally:
        ctx.close()
