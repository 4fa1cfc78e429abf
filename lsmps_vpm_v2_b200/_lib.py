"""ctypes binding of the C ABI in include/vpm_fmm.h (libvpm_fmm.so, built
in-tree by ``python -m lsmps_vpm_v2_b200.build``).

There is no fallback: if the shared library is missing or cannot be loaded,
every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
SO_PATH = os.path.join(HERE, "libvpm_fmm.so")

VPM_OK = 0
VPM_EDEVICE = 5
VPM_ENOMEM = 12
VPM_EINVAL = 22
VPM_EOVERFLOW = 75
VPM_ETIMEDOUT = 110

PREC_FP64 = 0
PREC_MIXED = 1
PREC_MIXED_FP64_M2L = 2
PREC_MIXED_TC = 3
BINOM_REFERENCE = 0
BINOM_EXACT = 1


class Params(C.Structure):
    """vpm_fmm_params (include/vpm_fmm.h)."""
    _fields_ = [
        ("p", C.c_int32),
        ("max_src", C.c_int32),
        ("max_par", C.c_int32),
        ("leaf_cap_3d", C.c_int32),
        ("exp_tree_pct", C.c_double),
        ("eps", C.c_double),
        ("precision", C.c_int32),
        ("binom", C.c_int32),
        ("max_depth", C.c_int32),
        ("use_graph", C.c_int32),
        ("center_3d", C.c_double * 3),
        ("support_3d", C.c_double),
    ]


class Stats(C.Structure):
    """vpm_fmm_stats (include/vpm_fmm.h)."""
    _fields_ = [
        ("n", C.c_int64),
        ("n_cells", C.c_int64),
        ("n_leaves", C.c_int64),
        ("min_level", C.c_int32),
        ("max_level", C.c_int32),
        ("p2p_pairs", C.c_int64),
        ("m2l_pairs", C.c_int64),
        ("m2p_pairs", C.c_int64),
        ("list1_len", C.c_int64),
        ("list3_len", C.c_int64),
        ("ms_tree", C.c_float),
        ("ms_lists", C.c_float),
        ("ms_upward", C.c_float),
        ("ms_m2l", C.c_float),
        ("ms_eval", C.c_float),
        ("ms_p2p", C.c_float),
        ("ms_total", C.c_float),
        ("kernels", C.c_int32),
        ("depth_retry", C.c_int32),
        ("ms_keys_sort", C.c_float),
        ("ms_levels", C.c_float),
        ("ms_l2l", C.c_float),
        ("pad_", C.c_float),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)

# name -> (restype, argtypes); every symbol declared in include/vpm_fmm.h.
SIGNATURES = {
    "vpm_fmm_params_default": (None, [C.POINTER(Params)]),
    "vpm_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "vpm_ctx_destroy": (C.c_int, [_vp]),
    "vpm_ctx_set_stream": (C.c_int, [_vp, _vp]),
    "vpm_ctx_sync": (C.c_int, [_vp]),
    "vpm_last_error": (C.c_char_p, [_vp]),
    "vpm_fmm2d_field": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int64, C.POINTER(Params), _vp, _vp,
                                  C.POINTER(Stats)]),
    "vpm_fmm2d_potential": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int64, C.POINTER(Params), _vp,
                                      C.POINTER(Stats)]),
    "vpm_fmm2d_field_device": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int64, C.POINTER(Params), _vp, _vp]),
    "vpm_velocity2d": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, C.c_int64, C.POINTER(Params), C.c_double,
                                 C.c_double, _vp, _vp, C.POINTER(Stats)]),
    "vpm_tree2d_build": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int64, C.POINTER(Params), C.POINTER(Stats)]),
    "vpm_last_stats": (C.c_int, [_vp, C.POINTER(Stats)]),
    "vpm_tree2d_counts": (C.c_int, [_vp, _i64p, _i64p, _i64p]),
    "vpm_tree2d_cells": (C.c_int, [_vp, _vp, _vp, _vp]),
    "vpm_tree2d_leaves": (C.c_int, [_vp, _vp, _vp, _vp]),
    "vpm_tree2d_list": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
    "vpm_measure_fma_peaks": (C.c_int, [_vp, _dp, _dp]),
    "vpm_measure_rcp_peak": (C.c_int, [_vp, _dp]),
    "vpm_stage_history": (C.c_int, [_vp, C.c_int32, C.c_int32, _vp, C.POINTER(C.c_int32)]),
    "vpm_fmm2d_field_batched": (C.c_int, [_vp, C.c_int32, _vp, _vp, _vp, _vp, _vp, C.POINTER(Params), _vp, _vp]),
    "vpm_batch_streams": (C.c_int, [_vp, _vp]),
    "vpm_fmm2d_field_batched_device": (C.c_int, [_vp, C.c_int32, _vp, _vp, _vp, _vp, _vp, C.POINTER(Params), _vp,
                                                 _vp]),
    "vpm_mlp_param_count": (C.c_int64, []),
    "vpm_selector_candidates": (C.c_int, [_vp, _vp, C.c_int32]),
    "vpm_mlp_init": (C.c_int, [_vp, C.c_uint64]),
    "vpm_mlp_set_params": (C.c_int, [_vp, _vp, C.c_int64]),
    "vpm_mlp_get_params": (C.c_int, [_vp, _vp, C.c_int64]),
    "vpm_mlp_set_norm": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "vpm_mlp_forward": (C.c_int, [_vp, _vp, C.c_int32, _vp, C.c_int32]),
    "vpm_mlp_grads": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int32, _vp, C.POINTER(C.c_float)]),
    "vpm_mlp_train": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int64, C.c_int32, C.c_int32, C.c_float, C.c_uint64, _vp]),
    "vpm_selector_features2d": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int64, C.c_double, _vp]),
    "vpm_selector_features2d_device": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int64, C.c_double, _vp]),
    "vpm_select2d": (C.c_int, [_vp, _vp, C.c_double, C.c_double, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                               C.POINTER(C.c_int32), _vp]),
    "vpm_direct3d_velocity_device": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int64, _vp, C.c_int64,
                                              _vp, _vp, _vp]),
    "vpm_direct2d_field_device": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int64, _vp, C.c_int64, _vp, _vp]),
    "vpm_fmm3d_velocity": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int64, C.POINTER(Params),
                                     _vp, _vp, _vp, C.POINTER(Stats)]),
    "vpm_fmm3d_velocity_device": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int64, C.POINTER(Params),
                                            _vp, _vp, _vp]),
    "vpm_velocity3d": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int64, C.POINTER(Params),
                                 C.c_double, C.c_double, C.c_double, _vp, _vp, _vp, C.POINTER(Stats)]),
    "vpm_tree3d_build": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int64, C.POINTER(Params), C.POINTER(Stats)]),
    "vpm_tree3d_counts": (C.c_int, [_vp, _i64p, _i64p, _i32p]),
    "vpm_tree3d_cells": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "vpm_fmm3d_velocity_treecell": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int64,
                                              C.POINTER(Params), _vp, _vp, _vp, C.POINTER(Stats)]),
    "vpm_fmm3d_velocity_treecell_device": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int64,
                                                     C.POINTER(Params), _vp, _vp, _vp]),
    "vpm_treecell3d_build": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int64, C.POINTER(Params), C.POINTER(Stats)]),
    "vpm_tree3d_cell_ids": (C.c_int, [_vp, _vp]),
    "vpm_fmm2d_field_device_static": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int64, C.POINTER(Params), _vp, _vp, _vp,
                                                C.c_char_p, C.c_size_t]),
}

_LIB = None


def lib() -> C.CDLL:
    """The loaded product library (raises when it is missing)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(SO_PATH):
            raise RuntimeError(f"{SO_PATH} is missing: build it with `python -m lsmps_vpm_v2_b200.build`")
        L = C.CDLL(SO_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def default_params(**over) -> Params:
    p = Params()
    lib().vpm_fmm_params_default(C.byref(p))
    for k, v in over.items():
        setattr(p, k, v)
    return p


def treecell3d_params(**over) -> Params:
    """Defaults with the reference's 3D TreeCell leaf caps: at most 30 active
    and 50 particles per leaf (global.cpp:778-779)."""
    return default_params(max_src=30, max_par=50, **over)


class VpmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status
