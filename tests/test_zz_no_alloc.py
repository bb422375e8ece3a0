"""its_marching_cubes_noalloc: marching cubes for callers that cannot allocate device memory
while they run (for example work replayed inside a CUDA graph they captured themselves, or a
frame loop under a fixed memory budget). Its scan scratch is a fixed file-scope device array,
so it must return exactly what the allocating its_marching_cubes returns, on consecutive
calls that reuse that array. This file is collected last on purpose."""
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


@pytest.mark.gpu
def test_noalloc_marching_cubes_matches_allocating_entry_point():
    import torch
    from its_b200 import Context, lib
    L = lib()
    L.its_marching_cubes_noalloc.restype = C.c_int
    L.its_marching_cubes_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                                             C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]
    ctx = Context(0)
    try:
        R = 96
        field_h, o, w = _fitted_field(ctx, R)
        field = torch.from_numpy(field_h).cuda()
        po, pw = o.ctypes.data_as(C.c_void_p), w.ctypes.data_as(C.c_void_p)
        ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        for iso in (float(np.quantile(field_h, 0.3)), 0.0):
            n_ref = C.c_int64(0)
            ctx.check(L.its_marching_cubes(ctx.h, ptr(field), R, po, pw, iso, None, None, 0, C.byref(n_ref)), "mc")
            assert n_ref.value > 0
            cube_ref = torch.zeros(R ** 3, dtype=torch.uint8, device="cuda")
            tri_ref = torch.zeros(3 * n_ref.value, dtype=torch.float64, device="cuda")
            ctx.check(L.its_marching_cubes(ctx.h, ptr(field), R, po, pw, iso, ptr(cube_ref), ptr(tri_ref),
                                           n_ref.value, C.byref(n_ref)), "mc")
            for _ in range(2):  # two calls in a row through the shared scratch array
                n = C.c_int64(-1)
                cube = torch.full((R ** 3,), 255, dtype=torch.uint8, device="cuda")
                tri = torch.full((3 * n_ref.value,), np.nan, dtype=torch.float64, device="cuda")
                ctx.check(L.its_marching_cubes_noalloc(ctx.h, ptr(field), R, po, pw, iso, ptr(cube), ptr(tri),
                                                       n_ref.value, C.byref(n)), "mc noalloc")
                assert n.value == n_ref.value
                assert torch.equal(cube, cube_ref)
                assert torch.equal(tri, tri_ref)  # tolerance: bit-exact, as the allocating path
        # limits: sizes beyond the fixed scratch and host buffers are refused
        n = C.c_int64(0)
        big = torch.zeros(1, dtype=torch.float64, device="cuda")
        assert L.its_marching_cubes_noalloc(ctx.h, ptr(big), 257, po, pw, 0.0, None, None, 0, C.byref(n)) == 1
        assert L.its_marching_cubes_noalloc(ctx.h, field_h.ctypes.data_as(C.c_void_p), R, po, pw, 0.0, None, None, 0,
                                            C.byref(n)) == 1
    finally:
        ctx.close()
