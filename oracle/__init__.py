"""CPU oracle for the ITS thin-shell path -- TEST INFRASTRUCTURE ONLY.

A C++ restatement of the reference algorithm (see orc_common.hpp for what it follows
and how far its parity is pinned), loaded through ctypes. Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may import this package, and
only as the checker or as the timed CPU baseline; the product never calls it.
"""
import ctypes as C
import os

import numpy as np

from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            path = _build.build()
        _lib = C.CDLL(path)
        _declare(_lib)
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _declare(L):
    vp, i64, i32, dbl = C.c_void_p, C.c_int64, C.c_int, C.c_double
    sig = {
        "orc_model_to_unit_cube": (None, [vp, i64, dbl]),
        "orc_uniform_bbox": (None, [vp, i64, vp, vp, vp]),
        "orc_tri_attributes": (None, [vp, vp, i64, vp, vp, vp]),
        "orc_morton_encode": (None, [vp, i64, vp]),
        "orc_morton_decode": (None, [vp, i64, vp]),
        "orc_luts": (None, [vp, vp, vp, vp]),
        "orc_hat": (None, [vp, vp, vp, i64, vp, vp]),
        "orc_svo_build": (vp, [vp, i64, vp, i64, i32, vp, vp]),
        "orc_svo_free": (None, [vp]),
        "orc_svo_counts": (None, [vp, vp]),
        "orc_svo_depth_counts": (None, [vp, vp, vp]),
        "orc_svo_voxels": (None, [vp, vp]),
        "orc_svo_nodes": (None, [vp, vp, vp, vp, vp, vp, vp, vp]),
        "orc_svo_vertices": (None, [vp, vp, vp]),
        "orc_svo_edges": (None, [vp, vp, vp, vp]),
        "orc_assemble": (vp, [vp]),
        "orc_csr_rows": (i64, [vp]),
        "orc_csr_nnz": (i64, [vp]),
        "orc_csr_get": (None, [vp, vp, vp, vp]),
        "orc_csr_from": (vp, [i64, vp, vp, vp]),
        "orc_csr_free": (None, [vp]),
        "orc_cgls": (i32, [vp, vp, vp, dbl, i64, i32, vp]),
        "orc_exact_start": (None, [vp, vp, vp, vp, vp]),
        "orc_exact_start_surplus": (None, [vp, vp, vp, vp, vp]),
        "orc_point_gradient": (None, [vp, vp, vp, vp, i64, vp, vp, vp, vp, vp]),
        "orc_intersections": (vp, [vp, vp, i64, vp, i64]),
        "orc_points_count": (i64, [vp, vp]),
        "orc_points_get": (None, [vp, vp]),
        "orc_points_free": (None, [vp]),
        "orc_signed_distance": (None, [vp, i64, vp, vp, i64, vp]),
        "orc_signed_distance_bvh": (None, [vp, i64, vp, vp, i64, vp]),
        "orc_cubic_assemble": (vp, [vp, vp, i64]),
        "orc_cubic_eval": (None, [vp, vp, vp, i64, vp]),
        "orc_cubic_eval_grid": (None, [vp, vp, vp, vp, i32, vp]),
        "orc_offset_samples": (None, [vp, i64, vp, i64, dbl, vp, vp]),
        "orc_bspline3": (None, [vp, i64, vp]),
        "orc_eval_points": (None, [vp, vp, vp, i64, vp, vp]),
        "orc_eval_brute": (None, [vp, vp, vp, i64, vp]),
        "orc_eval_grid": (None, [vp, vp, vp, vp, i32, vp]),
        "orc_marching_cubes": (i64, [vp, i32, vp, vp, dbl, vp, vp, i64]),
        "orc_point_query": (None, [vp, vp, vp, i64, vp, vp, dbl, dbl, vp, vp]),
        "orc_marching_cubes_mesh": (None, [vp, i32, vp, vp, dbl, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.reshape(shape) if shape is not None else a


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def model_to_unit_cube(V, scale=1.0):
    V = _f64(V).copy()
    lib().orc_model_to_unit_cube(_p(V), V.shape[0], scale)
    return V


def uniform_bbox(V):
    V = _f64(V)
    o, e, w = np.zeros(3), np.zeros(3), np.zeros(3)
    lib().orc_uniform_bbox(_p(V), V.shape[0], _p(o), _p(e), _p(w))
    return o, e, w


def tri_attributes(V, F):
    V, F = _f64(V), _i32(F)
    n = np.zeros((F.shape[0], 3)), np.zeros(F.shape[0]), np.zeros(F.shape[0])
    lib().orc_tri_attributes(_p(V), _p(F), F.shape[0], _p(n[0]), _p(n[1]), _p(n[2]))
    return n


def morton_encode(xyz):
    xyz = np.ascontiguousarray(xyz, dtype=np.uint32)
    out = np.zeros(xyz.shape[0], np.uint32)
    lib().orc_morton_encode(_p(xyz), xyz.shape[0], _p(out))
    return out


def morton_decode(m):
    m = np.ascontiguousarray(m, dtype=np.uint32)
    out = np.zeros((m.shape[0], 3), np.uint32)
    lib().orc_morton_decode(_p(m), m.shape[0], _p(out))
    return out


def luts():
    p, c = np.zeros((8, 27), np.int16), np.zeros((8, 27), np.int16)
    v, e = np.zeros(64, np.int16), np.zeros(48, np.int16)
    lib().orc_luts(_p(p), _p(c), _p(v), _p(e))
    return p, c, v, e


def hat(p, w, q):
    """Hat value and gradient of the corner at p (width w) at the points q (BSpline.hpp:4-57)."""
    p, q, w = _f64(p, (-1, 3)), _f64(q, (-1, 3)), _f64(w)
    val, grad = np.zeros(p.shape[0]), np.zeros((p.shape[0], 3))
    lib().orc_hat(_p(p), _p(w), _p(q), p.shape[0], _p(val), _p(grad))
    return val, grad


class Svo:
    """Oracle octree: ThinShells' SparseVoxelOctree restated on the CPU."""

    def __init__(self, V, F, res, origin, width):
        self.V, self.F = _f64(V), _i32(F)
        o, w = _f64(origin), _f64(width)
        self.h = lib().orc_svo_build(_p(self.V), self.V.shape[0], _p(self.F), self.F.shape[0], res, _p(o), _p(w))
        c = np.zeros(6, np.int64)
        lib().orc_svo_counts(self.h, _p(c))
        self.depth, self.num_voxels, self.num_fine, self.num_nodes, self.num_verts, self.num_edges = map(int, c)
        self.res, self.origin, self.width = res, o, w

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_svo_free(self.h)
            self.h = None

    def depth_counts(self):
        n, v = np.zeros(self.depth, np.int64), np.zeros(self.depth, np.int64)
        lib().orc_svo_depth_counts(self.h, _p(n), _p(v))
        return n, v

    def voxels(self):
        out = np.zeros(self.num_voxels, np.uint32)
        lib().orc_svo_voxels(self.h, _p(out))
        return out

    def nodes(self):
        N = self.num_nodes
        r = dict(morton=np.zeros(N, np.uint32), parent=np.zeros(N, np.uint32),
                 childs=np.zeros((N, 8), np.uint32), is_leaf=np.zeros(N, np.uint8),
                 origin=np.zeros((N, 3)), width=np.zeros(N), neighbors=np.zeros((N, 27), np.uint32))
        lib().orc_svo_nodes(self.h, _p(r["morton"]), _p(r["parent"]), _p(r["childs"]), _p(r["is_leaf"]),
                            _p(r["origin"]), _p(r["width"]), _p(r["neighbors"]))
        return r

    def vertices(self):
        pos, own = np.zeros((self.num_verts, 3)), np.zeros(self.num_verts, np.uint32)
        lib().orc_svo_vertices(self.h, _p(pos), _p(own))
        return pos, own

    def edges(self):
        E = self.num_edges
        p0, p1, own = np.zeros((E, 3)), np.zeros((E, 3)), np.zeros(E, np.uint32)
        lib().orc_svo_edges(self.h, _p(p0), _p(p1), _p(own))
        return p0, p1, own

    def assemble(self):
        h = lib().orc_assemble(self.h)
        try:
            n, nnz = lib().orc_csr_rows(h), lib().orc_csr_nnz(h)
            rp, col, val = np.zeros(n + 1, np.int64), np.zeros(nnz, np.int32), np.zeros(nnz)
            lib().orc_csr_get(h, _p(rp), _p(col), _p(val))
        finally:
            lib().orc_csr_free(h)
        return rp, col, val

    def point_gradient(self, lam, P, box_origin, box_end, before=None):
        """Field, gradient and missing flags (ThinShells::getPointValGradient)."""
        lam, P = _f64(lam), _f64(P)
        m = P.shape[0]
        val, grad, miss = np.zeros(m), np.zeros((m, 3)), np.zeros(m, np.uint8)
        bo, be = _f64(box_origin), _f64(box_end)
        bf = None if before is None else _f64(before)
        lib().orc_point_gradient(self.h, _p(lam), _p(P), _p(bf), m, _p(bo), _p(be), _p(val), _p(grad), _p(miss))
        return val, grad, miss

    def exact_start(self, b, shares=None, form="explicit"):
        """Exact solution of A lambda = b for this octree's operator (shares: coefficients of
        the vertices coincident with a coarser corner, default 0). form "explicit": each
        surplus from G = b - finer shares (orc_exact_start); "surplus": the sequential
        coarse-to-fine definition (orc_exact_start_surplus)."""
        rp, col, val = self.assemble()
        b = _f64(b)
        h = lib().orc_csr_from(rp.shape[0] - 1, _p(rp), _p(col), _p(val))
        out = np.zeros(rp.shape[0] - 1)
        sh = None if shares is None else _f64(shares)
        fn = lib().orc_exact_start if form == "explicit" else lib().orc_exact_start_surplus
        try:
            fn(self.h, h, _p(b), _p(sh), _p(out))
        finally:
            lib().orc_csr_free(h)
        return out

    def intersections(self):
        h = lib().orc_intersections(self.h, _p(self.V), self.V.shape[0], _p(self.F), self.F.shape[0])
        try:
            ne = C.c_int64(0)
            n = lib().orc_points_count(h, C.byref(ne))
            out = np.zeros((n, 3))
            lib().orc_points_get(h, _p(out))
        finally:
            lib().orc_points_free(h)
        return out, int(ne.value)

    def eval_points(self, lam, P):
        lam, P = _f64(lam), _f64(P)
        out, miss = np.zeros(P.shape[0]), np.zeros(P.shape[0], np.uint8)
        lib().orc_eval_points(self.h, _p(lam), _p(P), P.shape[0], _p(out), _p(miss))
        return out, miss

    def eval_brute(self, lam, P):
        lam, P = _f64(lam), _f64(P)
        out = np.zeros(P.shape[0])
        lib().orc_eval_brute(self.h, _p(lam), _p(P), P.shape[0], _p(out))
        return out

    def point_query(self, lam, P, box_origin, box_end, inner, outer):
        lam, P = _f64(lam), _f64(P)
        vals, labels = np.zeros(P.shape[0]), np.zeros(P.shape[0], np.int8)
        lib().orc_point_query(self.h, _p(lam), _p(P), P.shape[0], _p(_f64(box_origin)), _p(_f64(box_end)),
                              float(inner), float(outer), _p(vals), _p(labels))
        return vals, labels

    def cubic_assemble(self, samples=None):
        """CSR of the cubic B-spline system: one row per corner vertex, then one per extra sample
        point; square, padded with empty columns past the last vertex."""
        S = np.zeros((0, 3)) if samples is None else _f64(samples, (-1, 3))
        h = lib().orc_cubic_assemble(self.h, _p(S), S.shape[0])
        try:
            n, nnz = lib().orc_csr_rows(h), lib().orc_csr_nnz(h)
            rp, col, val = np.zeros(n + 1, np.int64), np.zeros(nnz, np.int32), np.zeros(nnz)
            lib().orc_csr_get(h, _p(rp), _p(col), _p(val))
        finally:
            lib().orc_csr_free(h)
        return rp, col, val

    def cubic_eval(self, lam, P):
        lam, P = _f64(lam), _f64(P, (-1, 3))
        out = np.zeros(P.shape[0])
        lib().orc_cubic_eval(self.h, _p(lam), _p(P), P.shape[0], _p(out))
        return out

    def cubic_eval_grid(self, lam, origin, width, R):
        lam = _f64(lam)
        out = np.zeros((R + 1) ** 3)
        lib().orc_cubic_eval_grid(self.h, _p(lam), _p(_f64(origin)), _p(_f64(width)), R, _p(out))
        return out

    def eval_grid(self, lam, origin, width, R):
        lam = _f64(lam)
        out = np.zeros((R + 1) ** 3)
        lib().orc_eval_grid(self.h, _p(lam), _p(_f64(origin)), _p(_f64(width)), R, _p(out))
        return out


def cgls(rowptr, col, val, b, tol, max_iters, stop=0, x0=None):
    """Eigen-semantics LSCG on a CSR matrix. Returns (x, report dict)."""
    rowptr = np.ascontiguousarray(rowptr, np.int64)
    col, val, b = np.ascontiguousarray(col, np.int32), _f64(val), _f64(b)
    n = rowptr.shape[0] - 1
    h = lib().orc_csr_from(n, _p(rowptr), _p(col), _p(val))
    x = np.zeros(n) if x0 is None else _f64(x0).copy()
    rep = np.zeros(5)
    try:
        lib().orc_cgls(h, _p(b), _p(x), tol, max_iters, stop, _p(rep))
    finally:
        lib().orc_csr_free(h)
    return x, dict(iterations=int(rep[0]), converged=bool(rep[1]), breakdown=bool(rep[2]),
                   rel_residual=float(rep[3]), normal_rel_residual=float(rep[4]))


def signed_distance(P, V, F):
    P, V, F = _f64(P), _f64(V), _i32(F)
    out = np.zeros(P.shape[0])
    lib().orc_signed_distance(_p(P), P.shape[0], _p(V), _p(F), F.shape[0], _p(out))
    return out


def signed_distance_bvh(P, V, F):
    """The signed distance as libits computes it: linear BVH, exact distance, fast winding number."""
    P, V, F = _f64(P), _f64(V), _i32(F)
    out = np.zeros(P.shape[0])
    lib().orc_signed_distance_bvh(_p(P), P.shape[0], _p(V), _p(F), F.shape[0], _p(out))
    return out


def offset_samples(V, F, eps):
    """Offset shell samples (v + eps n, then v - eps n, n the unit area-weighted vertex normal)
    and their targets (+eps, -eps)."""
    V, F = _f64(V), _i32(F)
    nv = V.shape[0]
    pts, tgt = np.zeros((2 * nv, 3)), np.zeros(2 * nv)
    lib().orc_offset_samples(_p(V), nv, _p(F), F.shape[0], float(eps), _p(pts), _p(tgt))
    return pts, tgt


def bspline3(t):
    t = _f64(t)
    out = np.zeros(t.shape[0])
    lib().orc_bspline3(_p(t), t.shape[0], _p(out))
    return out


def marching_cubes_mesh(field, R, origin, width, iso):
    field = _f64(field)
    cnt = np.zeros(2, np.int64)
    o, w = _f64(origin), _f64(width)
    lib().orc_marching_cubes_mesh(_p(field), R, _p(o), _p(w), iso, None, None, _p(cnt))
    verts, tris = np.zeros((max(cnt[0], 1), 3)), np.zeros((max(cnt[1], 1), 3), np.int32)
    lib().orc_marching_cubes_mesh(_p(field), R, _p(o), _p(w), iso, _p(verts), _p(tris), _p(cnt))
    return verts[:cnt[0]], tris[:cnt[1]]


def marching_cubes(field, R, origin, width, iso, with_triangles=True):
    field = _f64(field)
    cube = np.zeros(R ** 3, np.uint8)
    total = lib().orc_marching_cubes(_p(field), R, _p(_f64(origin)), _p(_f64(width)), iso, _p(cube), None, 0)
    tri = None
    if with_triangles:
        tri = np.zeros((max(total, 1), 3))
        lib().orc_marching_cubes(_p(field), R, _p(_f64(origin)), _p(_f64(width)), iso, _p(cube), _p(tri), total)
        tri = tri[:total]
    return cube, tri, int(total)
