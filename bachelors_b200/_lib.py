"""ctypes bindings for libfmmcuda.so (the C ABI in include/fmmcuda.h).

The library is built in-tree by bachelors_b200/build.py. Loading fails loudly if it is
missing: there is no CPU fallback anywhere in the package.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfmmcuda.so")

FMM_OK, FMM_E_INVALID, FMM_E_OOM, FMM_E_CUDA, FMM_E_TIMEOUT, FMM_E_LIMIT = range(6)
FMM_FP32, FMM_FP64 = 0, 1
FMM_M2L_SIMT, FMM_M2L_BF16X3, FMM_M2L_TF32, FMM_M2L_BF16X6 = 0, 1, 2, 3
FMM_TREECODE_REFERENCE_NEAR, FMM_TREECODE_FD_CURL = 1, 2

# Every extern "C" symbol include/fmmcuda.h declares.
EXPORTS = [
    "fmm_default_config", "fmm_plan_create", "fmm_plan_destroy", "fmm_set_sources", "fmm_set_sources_async", "fmm_set_bem_sources",
    "fmm_set_targets",
    "fmm_set_targets_to_sources",
    "fmm_build_tree", "fmm_upward", "fmm_downward", "fmm_evaluate", "fmm_solve", "fmm_direct",
    "fmm_direct_fp64_subset", "fmm_treecode", "fmm_adjoint", "fmm_adjoint_direct", "fmm_autotune", "fmm_get_tuning",
    "fmm_set_tuning", "fmm_batch_set_coils", "fmm_batch_partition", "fmm_update_sources", "fmm_graph_capture", "fmm_graph_launch",
    "fmm_set_wait_limit", "fmm_get_stats", "fmm_get_operator", "fmm_direct_B_noalloc", "fmm_translate_all", "fmm_translate_all_matrix",
    "fmm_translate_all_matrix_complex", "fmm_torus_quadratures", "fmm_add_vectors",
    "fmm_last_error_string", "fmm_version",
]


class FmmConfig(ctypes.Structure):
    _fields_ = [
        ("order", ctypes.c_int),
        ("leaf_capacity", ctypes.c_int),
        ("target_leaf_capacity", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("m2l_mode", ctypes.c_int),
        ("m2l_truncate", ctypes.c_int),
        ("device", ctypes.c_int),
        ("root_center", ctypes.c_double * 3),
        ("root_half_width", ctypes.c_double),
        ("m2l_tc_degree_cutoff", ctypes.c_int),
    ]


class FmmStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("ms_tree", "ms_upward", "ms_m2l", "ms_downward", "ms_near", "ms_total")] + [
        (k, ctypes.c_int64)
        for k in ("nodes", "leaves", "levels", "v_pairs", "p2p_pairs", "p2p_interactions", "n_sources", "n_targets")
    ] + [("ms_adjoint", ctypes.c_double), ("coils", ctypes.c_int64), ("m2l_tiles", ctypes.c_int64),
         ("m2l_tile_offsets", ctypes.c_int64)]


class FmmTuning(ctypes.Structure):
    _fields_ = [("m2l_k_chunk", ctypes.c_int), ("near_tile", ctypes.c_int), ("p2m_chunk", ctypes.c_int),
                ("ms_upward", ctypes.c_double), ("ms_downward", ctypes.c_double), ("ms_near", ctypes.c_double)]


class FmmError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"fmmcuda status {status}: {message}")
        self.status = status


_lib = None


def load():
    """Loads libfmmcuda.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python bachelors_b200/build.py` "
                          "(the solver has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    i64 = ctypes.c_int64
    dbl = ctypes.c_double
    sig = {
        "fmm_default_config": (None, [ctypes.POINTER(FmmConfig)]),
        "fmm_plan_create": (ctypes.c_int, [ctypes.POINTER(FmmConfig), ctypes.POINTER(vp)]),
        "fmm_plan_destroy": (ctypes.c_int, [vp]),
        "fmm_set_sources": (ctypes.c_int, [vp, vp, vp, vp, i64, ctypes.c_int, vp]),
        "fmm_set_sources_async": (ctypes.c_int, [vp, vp, vp, vp, i64, vp]),
        "fmm_set_bem_sources": (ctypes.c_int, [vp, vp, vp, vp, vp, i64, ctypes.c_int, vp]),
        "fmm_set_targets": (ctypes.c_int, [vp, vp, i64, ctypes.c_int, vp]),
        "fmm_set_targets_to_sources": (ctypes.c_int, [vp, vp]),
        "fmm_build_tree": (ctypes.c_int, [vp, vp]),
        "fmm_upward": (ctypes.c_int, [vp, vp]),
        "fmm_downward": (ctypes.c_int, [vp, vp]),
        "fmm_evaluate": (ctypes.c_int, [vp, dbl, ctypes.c_int, vp, vp, ctypes.c_int, vp]),
        "fmm_solve": (ctypes.c_int, [vp, dbl, ctypes.c_int, vp, vp, ctypes.c_int, vp]),
        "fmm_direct": (ctypes.c_int, [vp, dbl, ctypes.c_int, vp, vp, ctypes.c_int, vp]),
        "fmm_direct_fp64_subset": (ctypes.c_int, [vp, dbl, vp, i64, vp]),
        "fmm_treecode": (ctypes.c_int, [vp, dbl, ctypes.c_int, vp, i64, vp, vp, ctypes.c_int, ctypes.c_int, vp]),
        "fmm_adjoint": (ctypes.c_int, [vp, dbl, vp, vp, vp, ctypes.c_int, vp]),
        "fmm_adjoint_direct": (ctypes.c_int, [vp, dbl, vp, vp, vp, ctypes.c_int, vp]),
        "fmm_autotune": (ctypes.c_int, [vp, ctypes.POINTER(FmmTuning), vp]),
        "fmm_get_tuning": (ctypes.c_int, [vp, ctypes.POINTER(FmmTuning)]),
        "fmm_set_tuning": (ctypes.c_int, [vp, ctypes.POINTER(FmmTuning)]),
        "fmm_batch_set_coils": (ctypes.c_int, [vp, i64, vp, vp]),
        "fmm_batch_partition": (ctypes.c_int, [i64, vp, vp, ctypes.c_int, vp]),
        "fmm_update_sources": (ctypes.c_int, [vp, vp, vp, ctypes.c_int, vp]),
        "fmm_graph_capture": (ctypes.c_int, [vp, ctypes.c_int, vp]),
        "fmm_graph_launch": (ctypes.c_int, [vp, dbl, vp, vp, ctypes.c_int, vp]),
        "fmm_set_wait_limit": (ctypes.c_int, [vp, dbl]),
        "fmm_get_stats": (ctypes.c_int, [vp, ctypes.POINTER(FmmStats)]),
        "fmm_get_operator": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, vp]),
        "fmm_direct_B_noalloc": (ctypes.c_int, [vp, vp, vp, i64, vp, i64, dbl, vp, vp]),
        "fmm_translate_all": (ctypes.c_int, [vp, vp, vp, i64, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]),
        "fmm_translate_all_matrix": (ctypes.c_int, [vp, vp, vp, i64, ctypes.c_int, i64, ctypes.c_int, ctypes.c_int,
                                                    vp]),
        "fmm_translate_all_matrix_complex": (ctypes.c_int, [vp, vp, vp, i64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                            vp]),
        "fmm_torus_quadratures": (ctypes.c_int, [dbl, dbl, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_int,
                                                 ctypes.c_int, vp, vp, ctypes.c_int, vp]),
        "fmm_add_vectors": (ctypes.c_int, [vp, vp, vp, i64]),
        "fmm_last_error_string": (ctypes.c_char_p, []),
        "fmm_version": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != FMM_OK:
        msg = load().fmm_last_error_string().decode(errors="replace")
        raise FmmError(status, msg)
