"""Python layer over the libits C ABI: contexts, octrees, operators and the solver.

Arrays may be numpy arrays (host) or torch CUDA tensors (device); results come back as
numpy arrays unless a device output is passed. Every entry point goes through libits.so.
"""
import ctypes as C
import mmap
import weakref

import numpy as np

from . import _lib
from ._lib import ItsError, SolveOpts, SolveReport, SvoInfo, lib

STOP_NORMAL, STOP_RESIDUAL = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
OP_FP64, OP_FP32_VALUES = 0, 1


def _host_array(shape, dtype=np.float64):
    """A zero-filled host array for a large result copied from the device. Large ones live in
    anonymous memory advised for transparent huge pages, so that the copy that first writes
    them takes one page fault per 2 MB instead of one per 4 KB; small ones are plain numpy."""
    dtype = np.dtype(dtype)
    count = int(np.prod(shape))
    nbytes = count * dtype.itemsize
    if nbytes < (8 << 20) or not hasattr(mmap, "MADV_HUGEPAGE"):
        return np.zeros(shape, dtype)
    huge = 2 << 20
    mm = mmap.mmap(-1, (nbytes + huge - 1) // huge * huge, flags=mmap.MAP_PRIVATE | mmap.MAP_ANONYMOUS)
    try:
        mm.madvise(mmap.MADV_HUGEPAGE)
    except OSError:
        pass
    return np.frombuffer(mm, dtype=dtype, count=count).reshape(shape)


def _ptr(a):
    """Raw pointer of a numpy array or a torch tensor (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(C.c_void_p)
    return C.c_void_p(a.data_ptr())  # torch tensor


def _f64(a):
    if isinstance(a, np.ndarray) or not hasattr(a, "data_ptr"):
        return np.ascontiguousarray(a, dtype=np.float64)
    import torch
    assert a.dtype is torch.float64 and a.is_contiguous()
    return a


def _i32(a):
    if isinstance(a, np.ndarray) or not hasattr(a, "data_ptr"):
        return np.ascontiguousarray(a, dtype=np.int32)
    assert str(a.dtype) == "torch.int32" and a.is_contiguous()
    return a


def _n(a):
    return int(a.shape[0])


class Context:
    """An its_ctx: one GPU, one stream."""

    def __init__(self, device=0):
        h = C.c_void_p()
        s = lib().its_create(C.byref(h), device)
        if s != 0:
            raise ItsError(s, "its_create(device=%d) failed" % device)
        self.h = h
        self.device = device
        self._L = lib()  # kept for close() at interpreter shutdown, when module globals are gone
        self._children = weakref.WeakSet()  # objects that must be freed before the context

    def check(self, s, what):
        if s != 0:
            raise ItsError(s, "%s: %s" % (what, lib().its_last_error(self.h).decode()))

    def _adopt(self, obj):
        self._children.add(obj)

    def close(self):
        """Free every octree/operator made on this context, then the context itself."""
        if getattr(self, "h", None):
            for obj in sorted(list(self._children), key=lambda o: 0 if type(o).__name__ == "Operator" else 1):
                obj.close()
            self._L.its_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_stream(self, stream_ptr):
        self.check(lib().its_set_stream(self.h, C.c_void_p(stream_ptr)), "its_set_stream")

    def synchronize(self):
        self.check(lib().its_synchronize(self.h), "its_synchronize")

    def set_autotune(self, enable=True, cache_path=None):
        """Pick launch shapes by measurement (its_set_autotune); choices persist in cache_path."""
        self.check(lib().its_set_autotune(self.h, 1 if enable else 0,
                                          None if cache_path is None else cache_path.encode()), "its_set_autotune")

    def to_device(self, a):
        """A torch CUDA tensor holding a copy of host array a (its_copy_to_device: large
        pageable arrays go through page-locked chunks filled by host threads)."""
        import torch
        a = np.ascontiguousarray(a)
        out = torch.empty(a.shape, dtype=getattr(torch, a.dtype.name), device="cuda")
        self.check(lib().its_copy_to_device(self.h, C.c_void_p(out.data_ptr()), a.ctypes.data_as(C.c_void_p),
                                            a.nbytes), "its_copy_to_device")
        return out

    def autotune_choices(self):
        n = C.c_int64(0)
        self.check(lib().its_autotune_choices(self.h, None, 0, C.byref(n)), "its_autotune_choices")
        buf = C.create_string_buffer(n.value + 1)
        self.check(lib().its_autotune_choices(self.h, buf, n.value + 1, C.byref(n)), "its_autotune_choices")
        return dict((k, int(v)) for k, v in (line.split() for line in buf.value.decode().splitlines() if line))

    @property
    def kernel_launches(self):
        return int(lib().its_kernel_launches(self.h))

    # ---- a3 / a10 / a15 -------------------------------------------------------------
    def tri_attributes(self, V, F):
        V, F = _f64(V), _i32(F)
        nf = _n(F)
        n, a, d = np.zeros((nf, 3)), np.zeros(nf), np.zeros(nf)
        self.check(lib().its_tri_attributes(self.h, _ptr(V), _n(V), _ptr(F), nf, _ptr(n), _ptr(a), _ptr(d)),
                   "its_tri_attributes")
        return n, a, d

    def signed_distance(self, P, V, F, out=None):
        P, V, F = _f64(P), _f64(V), _i32(F)
        if out is None:
            out = np.zeros(_n(P))
        self.check(lib().its_signed_distance(self.h, _ptr(P), _n(P), _ptr(V), _n(V), _ptr(F), _n(F), _ptr(out)),
                   "its_signed_distance")
        return out

    def offset_samples(self, V, F, eps):
        """Offset shell samples v + eps n, then v - eps n (n the unit area-weighted vertex
        normal), and their targets +eps / -eps (its_offset_samples)."""
        V, F = _f64(V), _i32(F)
        nv = _n(V)
        pts, tgt = np.zeros((2 * nv, 3)), np.zeros(2 * nv)
        self.check(lib().its_offset_samples(self.h, _ptr(V), nv, _ptr(F), _n(F), float(eps), _ptr(pts), _ptr(tgt)),
                   "its_offset_samples")
        return pts, tgt

    def marching_cubes(self, field, res, origin, width, iso, triangles=True):
        field = _f64(field)
        o, w = np.ascontiguousarray(origin, np.float64), np.ascontiguousarray(width, np.float64)
        cube = np.zeros(res ** 3, np.uint8)
        n = C.c_int64(0)
        self.check(lib().its_marching_cubes(self.h, _ptr(field), res, _ptr(o), _ptr(w), float(iso), _ptr(cube), None, 0,
                                            C.byref(n)), "its_marching_cubes")
        tri = None
        if triangles:
            tri = _host_array((max(n.value, 1), 3))
            self.check(lib().its_marching_cubes(self.h, _ptr(field), res, _ptr(o), _ptr(w), float(iso), None,
                                                _ptr(tri), n.value, C.byref(n)), "its_marching_cubes")
            tri = tri[:n.value]
        return cube, tri, int(n.value)


def _mc_mesh(ctx, field, res, origin, width, iso):
    field = _f64(field)
    o, w = np.ascontiguousarray(origin, np.float64), np.ascontiguousarray(width, np.float64)
    nv, nt = C.c_int64(0), C.c_int64(0)
    L = lib()
    ctx.check(L.its_marching_cubes_mesh(ctx.h, _ptr(field), res, _ptr(o), _ptr(w), float(iso), None, 0, C.byref(nv),
                                        None, 0, C.byref(nt)), "its_marching_cubes_mesh")
    verts, tris = np.zeros((max(nv.value, 1), 3)), np.zeros((max(nt.value, 1), 3), np.int32)
    ctx.check(L.its_marching_cubes_mesh(ctx.h, _ptr(field), res, _ptr(o), _ptr(w), float(iso), _ptr(verts), nv.value,
                                        C.byref(nv), _ptr(tris), nt.value, C.byref(nt)), "its_marching_cubes_mesh")
    return verts[:nv.value], tris[:nt.value]


Context.marching_cubes_mesh = _mc_mesh


def model_to_unit_cube(V, scale=1.0):
    V = np.ascontiguousarray(V, np.float64).copy()
    s = lib().its_model_to_unit_cube(_ptr(V), _n(V), scale)
    if s != 0:
        raise ItsError(s, "its_model_to_unit_cube")
    return V


def uniform_bbox(V):
    V = np.ascontiguousarray(V, np.float64)
    o, e, w = np.zeros(3), np.zeros(3), np.zeros(3)
    s = lib().its_uniform_bbox(_ptr(V), _n(V), _ptr(o), _ptr(e), _ptr(w))
    if s != 0:
        raise ItsError(s, "its_uniform_bbox")
    return o, e, w


class Svo:
    """An its_svo: the sparse voxel octree of one mesh (SparseVoxelOctree of the reference)."""

    def __init__(self, ctx, V, F, res, origin, width):
        self.ctx = ctx
        V, F = _f64(V), _i32(F)
        o, w = np.ascontiguousarray(origin, np.float64), np.ascontiguousarray(width, np.float64)
        h = C.c_void_p()
        ctx.check(lib().its_svo_build(ctx.h, _ptr(V), _n(V), _ptr(F), _n(F), res, _ptr(o), _ptr(w), C.byref(h)),
                  "its_svo_build")
        self.h = h
        ctx._adopt(self)
        info = SvoInfo()
        ctx.check(lib().its_svo_get_info(h, C.byref(info)), "its_svo_get_info")
        self.info = info
        self.depth = info.depth
        self.res = res
        self.num_voxels, self.num_fine = info.num_voxels, info.num_fine_nodes
        self.num_nodes, self.num_verts, self.num_edges = info.num_nodes, info.num_vertices, info.num_edges
        self.origin, self.width = o, w

    def close(self):
        if getattr(self, "h", None):
            if self.ctx.h is not None:  # a closed context has already freed its objects
                self.ctx._L.its_svo_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def point_gradient(self, lam, P, box_origin, box_end, before=None):
        """Field, gradient (n x 3) and missing flags (its_point_value_gradient)."""
        lam, P = _f64(lam), _f64(P)
        m = _n(P)
        val, grad, miss = np.zeros(m), np.zeros((m, 3)), np.zeros(m, np.uint8)
        bo, be = np.ascontiguousarray(box_origin, np.float64), np.ascontiguousarray(box_end, np.float64)
        bf = None if before is None else _f64(before)
        self.ctx.check(lib().its_point_value_gradient(self.h, _ptr(lam), _ptr(P), _ptr(bf), m, _ptr(bo), _ptr(be),
                                                      _ptr(val), _ptr(grad), _ptr(miss)), "its_point_value_gradient")
        return val, grad, miss

    def exact_start(self, b, shares=None, out=None):
        """Hierarchical-surplus exact solution of A lambda = b, matrix-free (its_exact_start)."""
        b = _f64(b)
        sh = None if shares is None else _f64(shares)
        if out is None:
            out = np.zeros(self.num_verts)
        self.ctx.check(lib().its_exact_start(self.h, _ptr(b), _ptr(sh), _ptr(out)), "its_exact_start")
        return out

    def residual(self, b, lam):
        """||b - A lambda|| / ||b|| without an assembled operator (its_fit_residual)."""
        b, lam = _f64(b), _f64(lam)
        rel = C.c_double(0)
        self.ctx.check(lib().its_fit_residual(self.h, _ptr(b), _ptr(lam), C.byref(rel)), "its_fit_residual")
        return rel.value

    def share_features(self, b, norm=None, out=None, ids=None):
        """Features of the share network (its_share_features): (features n x 64, vertex ids).

        out / ids may be preallocated (numpy or torch CUDA) with enough rows."""
        b = _f64(b)
        nrm = None if norm is None else np.ascontiguousarray(norm, np.float32)
        cnt = C.c_int64(0)
        L = lib()
        self.ctx.check(L.its_share_features(self.h, _ptr(b), _ptr(nrm), None, 0, None, C.byref(cnt)),
                       "its_share_features")
        n = cnt.value
        feats = out if out is not None else np.zeros((max(n, 1), 64), np.float32)
        idv = ids if ids is not None else np.zeros(max(n, 1), np.int64)
        cap = int(feats.shape[0])
        self.ctx.check(L.its_share_features(self.h, _ptr(b), _ptr(nrm), _ptr(feats), cap, _ptr(idv), C.byref(cnt)),
                       "its_share_features")
        return feats[:n], idv[:n]

    def depth_counts(self):
        return (np.array(self.info.nodes_per_depth[:self.depth], np.int64),
                np.array(self.info.vertices_per_depth[:self.depth], np.int64))

    def voxels(self):
        out = np.zeros(self.num_voxels, np.uint32)
        self.ctx.check(lib().its_svo_get_voxels(self.h, _ptr(out)), "its_svo_get_voxels")
        return out

    def nodes(self):
        N = self.num_nodes
        r = dict(morton=np.zeros(N, np.uint32), parent=np.zeros(N, np.uint32), childs=np.zeros((N, 8), np.uint32),
                 is_leaf=np.zeros(N, np.uint8), origin=np.zeros((N, 3)), width=np.zeros(N),
                 neighbors=np.zeros((N, 27), np.uint32))
        self.ctx.check(lib().its_svo_get_nodes(self.h, _ptr(r["morton"]), _ptr(r["parent"]), _ptr(r["childs"]),
                                               _ptr(r["is_leaf"]), _ptr(r["origin"]), _ptr(r["width"]),
                                               _ptr(r["neighbors"])), "its_svo_get_nodes")
        return r

    def vertices(self):
        pos, own = np.zeros((self.num_verts, 3)), np.zeros(self.num_verts, np.uint32)
        self.ctx.check(lib().its_svo_get_vertices(self.h, _ptr(pos), _ptr(own)), "its_svo_get_vertices")
        return pos, own

    def vertex_positions_device(self):
        """The corner vertices' positions as a torch CUDA tensor (n x 3), copied on the device."""
        import torch
        pos = torch.empty((self.num_verts, 3), dtype=torch.float64, device="cuda")
        self.ctx.check(lib().its_svo_get_vertices(self.h, _ptr(pos), None), "its_svo_get_vertices")
        return pos

    def edges(self):
        E = self.num_edges
        p0, p1, own = np.zeros((E, 3)), np.zeros((E, 3)), np.zeros(E, np.uint32)
        self.ctx.check(lib().its_svo_get_edges(self.h, _ptr(p0), _ptr(p1), _ptr(own)), "its_svo_get_edges")
        return p0, p1, own

    def shell_samples(self, V, F, device=False):
        """Shell samples (its_shell_samples): one call into a buffer sized for typical meshes
        (about one sample per face), a second only when the samples exceed it. device=True
        returns them in a torch CUDA tensor (V and F may be CUDA tensors as well)."""
        V, F = _f64(V), _i32(F)
        n, ne = C.c_int64(0), C.c_int64(0)
        cap = 2 * _n(F) + _n(V) + 1024
        if device:
            import torch
            out = torch.empty((cap, 3), dtype=torch.float64, device="cuda")
            self.ctx.check(lib().its_shell_samples(self.h, _ptr(V), _n(V), _ptr(F), _n(F), _ptr(out), cap, C.byref(n),
                                                   C.byref(ne)), "its_shell_samples")
            if n.value > cap:
                out = torch.empty((n.value, 3), dtype=torch.float64, device="cuda")
                self.ctx.check(lib().its_shell_samples(self.h, _ptr(V), _n(V), _ptr(F), _n(F), _ptr(out), n.value,
                                                       C.byref(n), C.byref(ne)), "its_shell_samples")
            return out[:n.value], int(ne.value)
        out = _host_array((cap, 3))
        self.ctx.check(lib().its_shell_samples(self.h, _ptr(V), _n(V), _ptr(F), _n(F), _ptr(out), cap, C.byref(n),
                                               C.byref(ne)), "its_shell_samples")
        if n.value > cap:
            out = _host_array((n.value, 3))
            self.ctx.check(lib().its_shell_samples(self.h, _ptr(V), _n(V), _ptr(F), _n(F), _ptr(out), n.value,
                                                   C.byref(n), C.byref(ne)), "its_shell_samples")
        return out[:n.value], int(ne.value)

    def eval_points(self, lam, P, out=None):
        lam, P = _f64(lam), _f64(P)
        m = _n(P)
        if out is None:
            out = np.zeros(m)
        miss = np.zeros(m, np.uint8)
        self.ctx.check(lib().its_eval_points(self.h, _ptr(lam), _ptr(P), m, _ptr(out), _ptr(miss)), "its_eval_points")
        return out, miss

    def shell_iso_values(self, lam, P):
        lam, P = _f64(lam), _f64(P)
        lo, hi, miss = C.c_double(0), C.c_double(0), C.c_int64(0)
        self.ctx.check(lib().its_shell_iso_values(self.h, _ptr(lam), _ptr(P), _n(P), C.byref(lo), C.byref(hi),
                                                  C.byref(miss)), "its_shell_iso_values")
        return lo.value, hi.value, int(miss.value)

    def point_query(self, lam, P, box_origin, box_end, inner, outer):
        """Values and in/shell/out labels (1 outside, -1 inside, 0 in the shell) of points."""
        lam, P = _f64(lam), _f64(P)
        m = _n(P)
        vals, labels = np.zeros(m), np.zeros(m, np.int8)
        bo, be = np.ascontiguousarray(box_origin, np.float64), np.ascontiguousarray(box_end, np.float64)
        self.ctx.check(lib().its_point_query(self.h, _ptr(lam), _ptr(P), m, _ptr(bo), _ptr(be), float(inner),
                                             float(outer), _ptr(vals), _ptr(labels)), "its_point_query")
        return vals, labels

    def eval_grid(self, lam, origin, width, res, out=None):
        lam = _f64(lam)
        o, w = np.ascontiguousarray(origin, np.float64), np.ascontiguousarray(width, np.float64)
        if out is None:
            out = _host_array((res + 1) ** 3)
        self.ctx.check(lib().its_eval_grid(self.h, _ptr(lam), _ptr(o), _ptr(w), res, _ptr(out)), "its_eval_grid")
        return out

    def eval_grid_f32(self, lam, origin, width, res, out=None):
        """FP32 dense field (its_eval_grid_f32)."""
        lam = _f64(lam)
        o, w = np.ascontiguousarray(origin, np.float64), np.ascontiguousarray(width, np.float64)
        if out is None:
            out = _host_array((res + 1) ** 3, np.float32)
        self.ctx.check(lib().its_eval_grid_f32(self.h, _ptr(lam), _ptr(o), _ptr(w), res, _ptr(out)),
                       "its_eval_grid_f32")
        return out

    def eval_grid_fast(self, lam, origin, width, res, out=None, fp32=False):
        """Dense field by prolongation on a lattice aligned with the octree (its_eval_grid_fast,
        its_eval_grid_fast_f32); other lattices fall back to the point-by-point forms."""
        lam = _f64(lam)
        o, w = np.ascontiguousarray(origin, np.float64), np.ascontiguousarray(width, np.float64)
        if out is None:
            out = _host_array((res + 1) ** 3, np.float32 if fp32 else np.float64)
        fn = lib().its_eval_grid_fast_f32 if fp32 else lib().its_eval_grid_fast
        self.ctx.check(fn(self.h, _ptr(lam), _ptr(o), _ptr(w), res, _ptr(out)), "its_eval_grid_fast")
        return out

    def eval_points_cubic(self, lam, P, out=None):
        """Field of cubic-basis coefficients at points (its_eval_points_cubic)."""
        lam, P = _f64(lam), _f64(P)
        m = _n(P)
        if out is None:
            out = np.zeros(m)
        self.ctx.check(lib().its_eval_points_cubic(self.h, _ptr(lam), _ptr(P), m, _ptr(out)), "its_eval_points_cubic")
        return out

    def eval_grid_cubic(self, lam, origin, width, res, out=None):
        """Field of cubic-basis coefficients on the (res+1)^3 lattice (its_eval_grid_cubic)."""
        lam = _f64(lam)
        o, w = np.ascontiguousarray(origin, np.float64), np.ascontiguousarray(width, np.float64)
        if out is None:
            out = _host_array((res + 1) ** 3)
        self.ctx.check(lib().its_eval_grid_cubic(self.h, _ptr(lam), _ptr(o), _ptr(w), res, _ptr(out)),
                       "its_eval_grid_cubic")
        return out

    def grid_mc(self, lam, origin, width, res, isos, fast=False, triangles=True):
        """Field once on the device, then marching cubes at every iso level (its_eval_grid_mc,
        ThinShells::mcVisualization's driver). Returns one (num_verts x 3) soup per level (or the
        counts with triangles=False)."""
        lam = _f64(lam)
        o, w = np.ascontiguousarray(origin, np.float64), np.ascontiguousarray(width, np.float64)
        iso = np.ascontiguousarray(isos, np.float64)
        k = int(iso.shape[0])
        cnt = np.zeros(k, np.int64)
        L = lib()
        if not triangles:
            self.ctx.check(L.its_eval_grid_mc(self.h, _ptr(lam), _ptr(o), _ptr(w), res, 1 if fast else 0, _ptr(iso),
                                              k, None, None, _ptr(cnt)), "its_eval_grid_mc")
            return cnt
        # one call into buffers sized for a surface crossing the grid (12 vertices per R^2 and
        # level, pages committed only where written), a second only for levels that exceed them
        cap = np.full(k, 12 * res * res + 1024, np.int64)
        outs = [_host_array((int(c), 3)) for c in cap]
        P = (C.c_void_p * k)(*[o_.ctypes.data for o_ in outs])
        self.ctx.check(L.its_eval_grid_mc(self.h, _ptr(lam), _ptr(o), _ptr(w), res, 1 if fast else 0, _ptr(iso), k,
                                          P, _ptr(cap), _ptr(cnt)), "its_eval_grid_mc")
        if np.any(cnt > cap):
            outs = [_host_array((max(int(c), 1), 3)) for c in cnt]
            P = (C.c_void_p * k)(*[o_.ctypes.data for o_ in outs])
            cap = cnt.copy()
            self.ctx.check(L.its_eval_grid_mc(self.h, _ptr(lam), _ptr(o), _ptr(w), res, 1 if fast else 0, _ptr(iso),
                                              k, P, _ptr(cap), _ptr(cnt)), "its_eval_grid_mc")
        return [x[:int(c)] for x, c in zip(outs, cnt)]

    def vertex_sdf(self, V, F):
        """Right-hand side b: signed distance of every corner vertex (ThinShells::cpSDFOfTreeNodes)."""
        pos, _ = self.vertices()
        return self.ctx.signed_distance(pos, V, F)


class Operator:
    """An its_op: the assembled basis matrix A and its transpose.

    degree 1 is the reference's hat basis; degree 3 the cubic B-spline basis, optionally with
    extra sample rows (samples, m x 3) after the corner vertices' rows (its_operator_build_ex);
    such a system is square-padded: b and the solution then have rows entries."""

    def __init__(self, svo, mode=OP_FP64, degree=1, samples=None):
        self.ctx, self.svo = svo.ctx, svo
        self.degree = degree
        h = C.c_void_p()
        if degree == 1 and samples is None:
            svo.ctx.check(lib().its_operator_build(svo.h, mode, C.byref(h)), "its_operator_build")
        else:
            from ._lib import BasisOpts
            S = None if samples is None else _f64(samples)
            opts = BasisOpts(degree, None if S is None else _ptr(S).value, 0 if S is None else _n(S))
            svo.ctx.check(lib().its_operator_build_ex(svo.h, mode, C.byref(opts), C.byref(h)), "its_operator_build_ex")
        self.h = h
        svo.ctx._adopt(self)
        r, z = C.c_int64(0), C.c_int64(0)
        svo.ctx.check(lib().its_operator_info(h, C.byref(r), C.byref(z)), "its_operator_info")
        self.rows, self.nnz = r.value, z.value

    def close(self):
        if getattr(self, "h", None):
            if self.ctx.h is not None:
                self.ctx._L.its_operator_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def csr(self):
        rp, col, val = np.zeros(self.rows + 1, np.int64), np.zeros(self.nnz, np.int32), np.zeros(self.nnz)
        self.ctx.check(lib().its_operator_get_csr(self.h, _ptr(rp), _ptr(col), _ptr(val)), "its_operator_get_csr")
        return rp, col, val

    def exact_start(self, b, shares=None, out=None):
        """Hierarchical-surplus exact solution of A lambda = b (its_exact_start on the octree)."""
        return self.svo.exact_start(b, shares, out)

    def apply(self, x, transpose=False, out=None):
        x = _f64(x)
        if out is None:
            out = np.zeros(self.rows)
        self.ctx.check(lib().its_operator_apply(self.h, _ptr(x), _ptr(out), 1 if transpose else 0), "its_operator_apply")
        return out

    def solve(self, b, tol=None, max_iters=0, stop_rule=STOP_NORMAL, precision=PREC_FP64, ir_steps=3,
              inner_tol=None, x0=None, check_every=0, out=None):
        """LSCG (Eigen semantics by default). Returns (lambda, report dict)."""
        opts = SolveOpts()
        lib().its_solve_opts_default(C.byref(opts))
        if tol is not None:
            opts.tol = tol
        opts.max_iters = max_iters
        opts.stop_rule, opts.precision, opts.ir_steps = stop_rule, precision, ir_steps
        if inner_tol is not None:
            opts.inner_tol = inner_tol
        if check_every:
            opts.check_every = check_every
        keep = None
        if x0 is not None:
            keep = _f64(x0)
            opts.x0 = _ptr(keep).value if isinstance(keep, np.ndarray) else keep.data_ptr()
        b = _f64(b)
        if out is None:
            out = np.zeros(self.rows)
        rep = SolveReport()
        self.ctx.check(lib().its_lscg_solve(self.h, _ptr(b), _ptr(out), C.byref(opts), C.byref(rep)), "its_lscg_solve")
        return out, dict(iterations=rep.iterations, converged=bool(rep.converged), breakdown=bool(rep.breakdown),
                         rel_residual=rep.rel_residual, normal_rel_residual=rep.normal_rel_residual, ms=rep.ms,
                         inner_iterations=rep.inner_iterations)


def solve_batch(ops, bs, tol=None, max_iters=0, stop_rule=STOP_NORMAL, check_every=0, x0s=None, outs=None):
    """Batched LSCG over independent operators of one context (its_lscg_solve_batch).

    Returns (list of lambdas, list of report dicts)."""
    count = len(ops)
    ctx = ops[0].ctx
    opts = SolveOpts()
    lib().its_solve_opts_default(C.byref(opts))
    if tol is not None:
        opts.tol = tol
    opts.max_iters, opts.stop_rule = max_iters, stop_rule
    if check_every:
        opts.check_every = check_every
    bs = [_f64(b) for b in bs]
    outs = outs if outs is not None else [np.zeros(op.rows) for op in ops]
    keep = None
    if x0s is not None:
        keep = [_f64(x) for x in x0s]
        xarr = (C.c_void_p * count)(*[_ptr(x).value if isinstance(x, np.ndarray) else x.data_ptr() for x in keep])
        opts.x0 = C.cast(xarr, C.c_void_p).value
    H = (C.c_void_p * count)(*[op.h.value for op in ops])
    B = (C.c_void_p * count)(*[_ptr(b).value if isinstance(b, np.ndarray) else b.data_ptr() for b in bs])
    X = (C.c_void_p * count)(*[_ptr(x).value if isinstance(x, np.ndarray) else x.data_ptr() for x in outs])
    reps = (SolveReport * count)()
    ctx.check(lib().its_lscg_solve_batch(H, count, B, X, C.byref(opts), reps), "its_lscg_solve_batch")
    out = [dict(iterations=r.iterations, converged=bool(r.converged), breakdown=bool(r.breakdown),
                rel_residual=r.rel_residual, normal_rel_residual=r.normal_rel_residual, ms=r.ms) for r in reps]
    del keep
    return outs, out


def _addr(a):
    """Address of a contiguous numpy array or a torch tensor (None -> NULL). A writable array's
    address through the buffer protocol: about half the time of reading it through ctypes."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if a.flags.writeable and a.size and a.flags.c_contiguous:
            return C.addressof(C.c_char.from_buffer(a))
        return a.ctypes.data
    return a.data_ptr()


def exact_start_batch(svos, bs, shares=None, outs=None):
    """Exact starts of many octrees of one context (its_exact_start_batch)."""
    count = len(svos)
    bs = [_f64(b) for b in bs]
    sh = None if shares is None else [None if x is None else _f64(x) for x in shares]
    outs = outs if outs is not None else [np.zeros(s.num_verts) for s in svos]
    H = (C.c_void_p * count)(*[s.h.value for s in svos])
    B = (C.c_void_p * count)(*[_addr(b) for b in bs])
    S = None if sh is None else (C.c_void_p * count)(*[_addr(x) for x in sh])
    X = (C.c_void_p * count)(*[_addr(x) for x in outs])
    svos[0].ctx.check(lib().its_exact_start_batch(H, count, B, S, X), "its_exact_start_batch")
    return outs


def fit_residual_batch(svos, bs, lams):
    """||b - A lambda|| / ||b|| per octree, matrix-free (its_fit_residual_batch)."""
    count = len(svos)
    bs, lams = [_f64(b) for b in bs], [_f64(x) for x in lams]
    H = (C.c_void_p * count)(*[s.h.value for s in svos])
    B = (C.c_void_p * count)(*[_addr(b) for b in bs])
    X = (C.c_void_p * count)(*[_addr(x) for x in lams])
    rel = np.zeros(count)
    svos[0].ctx.check(lib().its_fit_residual_batch(H, count, B, X, _ptr(rel)), "its_fit_residual_batch")
    return rel


def learned_start_batch(svos, net, bs, norm, outs=None):
    """Learned starts of many octrees of one context (its_learned_start_batch)."""
    count = len(svos)
    bs = [_f64(b) for b in bs]
    norm = np.ascontiguousarray(norm, np.float32)
    outs = outs if outs is not None else [np.zeros(s.num_verts) for s in svos]
    H = (C.c_void_p * count)(*[s.h.value for s in svos])
    B = (C.c_void_p * count)(*[_addr(b) for b in bs])
    X = (C.c_void_p * count)(*[_addr(x) for x in outs])
    svos[0].ctx.check(lib().its_learned_start_batch(H, count, net.h, B, _ptr(norm), X), "its_learned_start_batch")
    return outs


# The last FP32 normalisation array passed to learned_fit as it is (contiguous float32, no copy
# made) and its address: the fit is called again and again with the same one, and reading an
# array's address through ctypes costs more than the rest of the call's Python side.
_norm_seen = [None, 0]


def _norm_arg(norm):
    if _norm_seen[0] is norm:
        return norm, _norm_seen[1]
    a = np.ascontiguousarray(norm, np.float32)
    addr = a.ctypes.data
    if a is norm:
        _norm_seen[0], _norm_seen[1] = a, addr
    return a, addr


def learned_fit(svo, net, b, norm, tol, out=None):
    """The learned fit of one octree (its_learned_fit): learned start, FP64 residual check,
    plain LSCG from the start when the residual misses tol. Returns (lambda, report dict)."""
    b = _f64(b)
    norm, norm_addr = _norm_arg(norm)
    if out is None:
        out = np.zeros(svo.num_verts)
    rep = SolveReport()
    svo.ctx.check(lib().its_learned_fit(svo.h, net.h, _addr(b), norm_addr, tol, _addr(out), C.byref(rep)),
                  "its_learned_fit")
    return out, dict(iterations=rep.iterations, converged=bool(rep.converged), rel_residual=rep.rel_residual,
                     ms=rep.ms)


def _f32(a):
    if isinstance(a, np.ndarray) or not hasattr(a, "data_ptr"):
        return np.ascontiguousarray(a, dtype=np.float32)
    assert str(a.dtype) == "torch.float32" and a.is_contiguous()
    return a


def feature_tiles(X):
    """FP32 features (n x 64) as the network kernel's input tiles (its_mlp_forward_tiles_async):
    BF16 (round to nearest even), 128-row tiles of 128-byte rows, the 16-byte chunk c of row r
    at chunk position c ^ (r % 8). Returns a uint8 array of ceil(n / 128) * 16384 bytes."""
    X = np.ascontiguousarray(X, np.float32)
    n = X.shape[0]
    tiles = (n + 127) // 128
    bits = np.zeros((tiles * 128, 64), np.uint32)
    bits[:n] = X.view(np.uint32)
    bf = ((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16).astype(np.uint16)  # RN-even to BF16
    rows = bf.reshape(tiles * 128, 8, 8)  # [row][chunk][8 values]
    r = np.arange(tiles * 128)
    out = np.empty_like(rows)
    for c in range(8):
        out[r, c ^ (r % 8)] = rows[:, c]
    return out.reshape(-1).view(np.uint8)


class ShareNet:
    """The share network (its_mlp): predicts minimum-norm shares from 64 vertex features."""

    def __init__(self, ctx, batch=65536, params=None):
        self.ctx = ctx
        h = C.c_void_p()
        ctx.check(lib().its_mlp_create(ctx.h, batch, C.byref(h)), "its_mlp_create")
        self.h, self.batch = h, batch
        self.num_params = int(lib().its_mlp_num_params())
        ctx._adopt(self)
        if params is not None:
            self.set_params(params)

    def close(self):
        if getattr(self, "h", None):
            if self.ctx.h is not None:
                self.ctx._L.its_mlp_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_params(self, params):
        p = _f32(params)
        assert p.shape[0] == self.num_params
        self.ctx.check(lib().its_mlp_set_params(self.h, _ptr(p)), "its_mlp_set_params")

    def params(self):
        p = np.zeros(self.num_params, np.float32)
        self.ctx.check(lib().its_mlp_get_params(self.h, _ptr(p)), "its_mlp_get_params")
        return p

    def forward(self, X, out=None):
        X = _f32(X)
        n = _n(X)
        if out is None:
            out = np.zeros(n, np.float32)
        self.ctx.check(lib().its_mlp_forward(self.h, _ptr(X), n, _ptr(out)), "its_mlp_forward")
        return out

    def forward_async(self, X, out):
        """Predictions for device (torch CUDA) features into a device output, queued without waiting."""
        self.ctx.check(lib().its_mlp_forward_async(self.h, _ptr(X), _n(X), _ptr(out)), "its_mlp_forward_async")
        return out

    def forward_tiles_async(self, tiles, n, out, after_kernel=False):
        """Predictions for n rows from device input tiles (feature_tiles' layout) into a device
        output, queued without waiting (its_mlp_forward_tiles_async)."""
        self.ctx.check(lib().its_mlp_forward_tiles_async(self.h, _ptr(tiles), int(n), _ptr(out), 1 if after_kernel else 0),
                       "its_mlp_forward_tiles_async")
        return out

    def check(self):
        self.ctx.check(lib().its_mlp_check(self.h), "its_mlp_check")

    def forward_layers(self, X, out=None):
        X = _f32(X)
        n = _n(X)
        if out is None:
            out = np.zeros(n, np.float32)
        self.ctx.check(lib().its_mlp_forward_layers(self.h, _ptr(X), n, _ptr(out)), "its_mlp_forward_layers")
        return out

    def gradient(self, X, y):
        X, y = _f32(X), _f32(y)
        g = np.zeros(self.num_params, np.float32)
        loss = C.c_float(0)
        self.ctx.check(lib().its_mlp_gradient(self.h, _ptr(X), _ptr(y), _n(X), _ptr(g), C.byref(loss)),
                       "its_mlp_gradient")
        return g, float(loss.value)

    def train(self, X, y, steps, lr=1e-3, seed=0):
        X, y = _f32(X), _f32(y)
        curve = np.zeros(max(steps, 1), np.float32)
        self.ctx.check(lib().its_mlp_train(self.h, _ptr(X), _ptr(y), _n(X), steps, lr, seed, _ptr(curve)),
                       "its_mlp_train")
        return curve[:steps]
