"""ctypes binding of libits.so (the C ABI declared in include/its/its.h).

The library is the product: there is no Python or CPU fallback. If libits.so is missing
or cannot be loaded, every call raises.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libits.so")

ITS_OK, ITS_ERR_INVALID, ITS_ERR_CUDA, ITS_ERR_OOM, ITS_ERR_TIMEOUT, ITS_ERR_NOT_CONVERGED, ITS_ERR_STATE = range(7)
STATUS_NAMES = {0: "ITS_OK", 1: "ITS_ERR_INVALID", 2: "ITS_ERR_CUDA", 3: "ITS_ERR_OOM", 4: "ITS_ERR_TIMEOUT",
                5: "ITS_ERR_NOT_CONVERGED", 6: "ITS_ERR_STATE"}


class SvoInfo(C.Structure):
    _fields_ = [("res", C.c_int), ("depth", C.c_int), ("num_voxels", C.c_int64), ("num_fine_nodes", C.c_int64),
                ("num_nodes", C.c_int64), ("num_vertices", C.c_int64), ("num_edges", C.c_int64),
                ("nodes_per_depth", C.c_int64 * 16), ("vertices_per_depth", C.c_int64 * 16),
                ("origin", C.c_double * 3), ("unit", C.c_double * 3), ("build_ms", C.c_double),
                ("learned_tables_ms", C.c_double)]


class BasisOpts(C.Structure):
    _fields_ = [("degree", C.c_int), ("samples", C.c_void_p), ("num_samples", C.c_int64)]


class SolveOpts(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_iters", C.c_int64), ("stop_rule", C.c_int), ("precision", C.c_int),
                ("ir_steps", C.c_int), ("inner_tol", C.c_double), ("x0", C.c_void_p), ("check_every", C.c_int)]


class SolveReport(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("converged", C.c_int), ("breakdown", C.c_int),
                ("rel_residual", C.c_double), ("normal_rel_residual", C.c_double), ("ms", C.c_double),
                ("inner_iterations", C.c_int64)]


vp, i64, i32, dbl, st = C.c_void_p, C.c_int64, C.c_int, C.c_double, C.c_int
SIGNATURES = {
    "its_create": (st, [C.POINTER(vp), i32]),
    "its_destroy": (st, [vp]),
    "its_last_error": (C.c_char_p, [vp]),
    "its_set_stream": (st, [vp, vp]),
    "its_synchronize": (st, [vp]),
    "its_version": (C.c_char_p, []),
    "its_kernel_launches": (i64, [vp]),
    "its_check_division": (st, [vp, vp, vp, i64, C.POINTER(i64)]),
    "its_set_autotune": (st, [vp, i32, C.c_char_p]),
    "its_copy_to_device": (st, [vp, vp, vp, i64]),
    "its_autotune_choices": (st, [vp, C.c_char_p, i64, C.POINTER(i64)]),
    "its_model_to_unit_cube": (st, [vp, i64, dbl]),
    "its_uniform_bbox": (st, [vp, i64, vp, vp, vp]),
    "its_tri_attributes": (st, [vp, vp, i64, vp, i64, vp, vp, vp]),
    "its_svo_build": (st, [vp, vp, i64, vp, i64, i32, vp, vp, C.POINTER(vp)]),
    "its_svo_free": (st, [vp]),
    "its_svo_get_info": (st, [vp, C.POINTER(SvoInfo)]),
    "its_svo_get_voxels": (st, [vp, vp]),
    "its_svo_get_nodes": (st, [vp, vp, vp, vp, vp, vp, vp, vp]),
    "its_svo_get_vertices": (st, [vp, vp, vp]),
    "its_svo_get_edges": (st, [vp, vp, vp, vp]),
    "its_shell_samples": (st, [vp, vp, i64, vp, i64, vp, i64, C.POINTER(i64), C.POINTER(i64)]),
    "its_signed_distance": (st, [vp, vp, i64, vp, i64, vp, i64, vp]),
    "its_operator_build": (st, [vp, i32, C.POINTER(vp)]),
    "its_operator_free": (st, [vp]),
    "its_operator_info": (st, [vp, C.POINTER(i64), C.POINTER(i64)]),
    "its_operator_get_csr": (st, [vp, vp, vp, vp]),
    "its_operator_apply": (st, [vp, vp, vp, i32]),
    "its_solve_opts_default": (st, [C.POINTER(SolveOpts)]),
    "its_lscg_solve": (st, [vp, vp, vp, C.POINTER(SolveOpts), C.POINTER(SolveReport)]),
    "its_lscg_solve_batch": (st, [vp, i64, vp, vp, C.POINTER(SolveOpts), vp]),
    "its_exact_start": (st, [vp, vp, vp, vp]),
    "its_exact_start_batch": (st, [vp, i64, vp, vp, vp]),
    "its_mlp_create": (st, [vp, i64, C.POINTER(vp)]),
    "its_mlp_free": (st, [vp]),
    "its_mlp_num_params": (i64, []),
    "its_mlp_set_params": (st, [vp, vp]),
    "its_mlp_get_params": (st, [vp, vp]),
    "its_mlp_forward": (st, [vp, vp, i64, vp]),
    "its_mlp_forward_async": (st, [vp, vp, i64, vp]),
    "its_mlp_forward_tiles_async": (st, [vp, vp, i64, vp, C.c_int]),
    "its_mlp_check": (st, [vp]),
    "its_mlp_forward_layers": (st, [vp, vp, i64, vp]),
    "its_mlp_gradient": (st, [vp, vp, vp, i64, vp, vp]),
    "its_mlp_train": (st, [vp, vp, vp, i64, i64, C.c_float, C.c_uint64, vp]),
    "its_fit_residual": (st, [vp, vp, vp, C.POINTER(dbl)]),
    "its_fit_residual_batch": (st, [vp, i64, vp, vp, vp]),
    "its_share_features": (st, [vp, vp, vp, vp, i64, vp, C.POINTER(i64)]),
    "its_learned_start": (st, [vp, vp, vp, vp, vp]),
    "its_learned_start_batch": (st, [vp, i64, vp, vp, vp, vp]),
    "its_learned_fit": (st, [vp, vp, vp, vp, dbl, vp, C.POINTER(SolveReport)]),
    "its_eval_points": (st, [vp, vp, vp, i64, vp, vp]),
    "its_shell_iso_values": (st, [vp, vp, vp, i64, C.POINTER(dbl), C.POINTER(dbl), C.POINTER(i64)]),
    "its_eval_grid": (st, [vp, vp, vp, vp, i32, vp]),
    "its_point_query": (st, [vp, vp, vp, i64, vp, vp, dbl, dbl, vp, vp]),
    "its_point_value_gradient": (st, [vp, vp, vp, vp, i64, vp, vp, vp, vp, vp]),
    "its_marching_cubes": (st, [vp, vp, i32, vp, vp, dbl, vp, vp, i64, C.POINTER(i64)]),
    "its_marching_cubes_f32": (st, [vp, vp, i32, vp, vp, dbl, vp, vp, i64, C.POINTER(i64)]),
    "its_eval_grid_f32": (st, [vp, vp, vp, vp, i32, vp]),
    "its_eval_grid_fast": (st, [vp, vp, vp, vp, i32, vp]),
    "its_eval_grid_mc": (st, [vp, vp, vp, vp, i32, i32, vp, i32, vp, vp, vp]),
    "its_operator_build_ex": (st, [vp, i32, vp, C.POINTER(vp)]),
    "its_eval_points_cubic": (st, [vp, vp, vp, i64, vp]),
    "its_eval_grid_cubic": (st, [vp, vp, vp, vp, i32, vp]),
    "its_offset_samples": (st, [vp, vp, i64, vp, i64, dbl, vp, vp]),
    "its_eval_grid_fast_f32": (st, [vp, vp, vp, vp, i32, vp]),
    "its_marching_cubes_mesh": (st, [vp, vp, i32, vp, vp, dbl, vp, i64, C.POINTER(i64), vp, i64, C.POINTER(i64)]),
}

_lib = None


def lib():
    """Load libits.so and declare its signatures (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libits.so is not built (run __graft_entry__.build() or its_b200/build.py)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class ItsError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), msg))
        self.status = status
