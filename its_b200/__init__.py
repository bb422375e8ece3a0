"""its_b200: a B200 (sm_100a) implementation of the ITS thin-shell hot path.

The GPU work lives in libits.so (its_b200/csrc, C ABI in include/its/its.h); this package
is the Python host layer: the ctypes binding (_lib), an object API (api), the seeded
synthetic meshes (meshes) and the share network's training and evaluation (sharenet).
"""
from .api import (OP_FP32_VALUES, OP_FP64, PREC_FP64, PREC_MIXED, STOP_NORMAL, STOP_RESIDUAL, Context,  # noqa: F401
                  Operator, Svo, model_to_unit_cube, uniform_bbox)
from ._lib import ItsError, lib  # noqa: F401
