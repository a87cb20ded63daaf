"""ctypes binding of libkifmm2d.so (declarations in include/kifmm2d.h).

The library is built in place (``python -m pykifmm2d_b200.build``) and loaded
from this package's folder.  There is no fallback: if the library is missing
or does not load, importing the binding raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libkifmm2d.so")

OK = 0
ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_DEPTH, ERR_STATE, ERR_RANGE, ERR_UNSUPPORTED = 1, 2, 3, 4, 5, 6, 7
MEM_HOST, MEM_DEVICE = 0, 1
KERNEL_LAPLACE, KERNEL_MOD_HELMHOLTZ, KERNEL_HELMHOLTZ = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
E2C_DENSE, E2C_CIRCULANT = 0, 1
M2L_AUTO, M2L_FP32, M2L_BF16X3, M2L_FP16X3, M2L_FP64, M2L_INT8, M2L_INT8X4 = 0, 1, 2, 3, 4, 5, 6
MAX_LEVELS = 30
NOALLOC_MAX_POINTS = 1048576
PHASES = ["tree", "sort", "precompute", "p2m", "m2m", "m2l", "leaf", "targets", "l2l", "operators", "closure", "entries", "nodes"]


class KernelDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("reserved", ctypes.c_int32), ("k", ctypes.c_double)]


class Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("m2l", ctypes.c_int32), ("fix_bbox", ctypes.c_int32),
                ("radii", ctypes.c_int32), ("device", ctypes.c_int32), ("near_fp64", ctypes.c_int32),
                ("stream", ctypes.c_void_p), ("e2c", ctypes.c_int32), ("iscomplex", ctypes.c_int32),
                ("planned", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class TreeInfo(ctypes.Structure):
    _fields_ = [("n_points", ctypes.c_int64), ("levels", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("n_nodes", ctypes.c_int64), ("n_leaves", ctypes.c_int64), ("n_fake", ctypes.c_int64),
                ("n_xlist", ctypes.c_int64), ("n_outside", ctypes.c_int64), ("root_min", ctypes.c_double),
                ("root_max", ctypes.c_double), ("n_p2p_pairs", ctypes.c_int64), ("n_p2m_points", ctypes.c_int64),
                ("n_m2l_pairs", ctypes.c_int64), ("n_m2l_groups", ctypes.c_int64),
                ("nodes_per_level", ctypes.c_int64 * MAX_LEVELS), ("planned_bytes", ctypes.c_int64)]


class KifmmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"kifmm error {code}: {msg}")
        self.code = code


_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_SIGS = {
    "kifmm_default_options": (None, [ctypes.POINTER(Options)]),
    "kifmm_plan_create": (_i32, [ctypes.POINTER(KernelDesc), _i32, _i32, ctypes.POINTER(Options), ctypes.POINTER(_vp)]),
    "kifmm_build_tree": (_i32, [_vp, _vp, _vp, _i64, _i32]),
    "kifmm_precompute": (_i32, [_vp]),
    "kifmm_build_expansions": (_i32, [_vp, _vp, _i32]),
    "kifmm_evaluate_to_sources": (_i32, [_vp, _vp, _i32, _i32]),
    "kifmm_evaluate_to_points": (_i32, [_vp, _vp, _vp, _i64, _i32, _vp, _i32]),
    "kifmm_synchronize": (_i32, [_vp]),
    "kifmm_graph_capture": (_i32, [_vp, _vp, _vp, _i32]),
    "kifmm_graph_launch": (_i32, [_vp]),
    "kifmm_batch_capture": (_i32, [_vp, _i32, _vp, _vp, _i32, _vp, ctypes.POINTER(_vp)]),
    "kifmm_batch_launch": (_i32, [_vp]),
    "kifmm_batch_synchronize": (_i32, [_vp]),
    "kifmm_batch_info": (_i32, [_vp, _vp, _vp]),
    "kifmm_batch_destroy": (_i32, [_vp]),
    "kifmm_batch_set_draws": (_i32, [_vp, _vp, _vp]),
    "kifmm_batch_sums": (_i32, [_vp, _vp]),
    "kifmm_stream_create": (_i32, [_i32, ctypes.POINTER(_vp)]),
    "kifmm_stream_destroy": (_i32, [_vp]),
    "kifmm_fill_normal": (_i32, [_vp, _i64, ctypes.c_uint64, ctypes.c_uint64, _vp]),
    "kifmm_get_tree_info": (_i32, [_vp, ctypes.POINTER(TreeInfo)]),
    "kifmm_export_tree": (_i32, [_vp, _vp, _vp]),
    "kifmm_export_lists": (_i32, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "kifmm_plan_destroy": (_i32, [_vp]),
    "kifmm_last_error": (ctypes.c_char_p, []),
    "kifmm_direct_sum": (_i32, [ctypes.POINTER(KernelDesc), _vp, _vp, _vp, _i64, _vp, _i64, _vp, _i32, _i32]),
    "kifmm_kernel_matrix": (_i32, [ctypes.POINTER(KernelDesc), _vp, _vp, _i64, _vp, _vp, _i64, _vp, _i32, _i32]),
    "kifmm_kernel_apply": (_i32, [ctypes.POINTER(KernelDesc), _vp, _vp, _i64, _vp, _vp, _i64, _vp, _vp, _i32, _i32]),
    "kifmm_set_profiling": (_i32, [_vp, _i32]),
    "kifmm_get_phase_times": (_i32, [_vp, _vp, _vp, _i32]),
    "kifmm_launch_count": (_i64, []),
    "kifmm_set_wait_limit": (_i32, [_vp, _i64]),
    "kifmm_morton_sort_noalloc": (_i32, [_vp, _vp, _i64, ctypes.c_double, ctypes.c_double, _vp, _vp, _vp]),
    "kifmm_version": (_i32, []),
}

_lib = None


def load():
    """Load libkifmm2d.so (raises if it is missing: no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m pykifmm2d_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def check(code):
    if code != OK:
        msg = load().kifmm_last_error()
        raise KifmmError(code, msg.decode() if msg else "")
