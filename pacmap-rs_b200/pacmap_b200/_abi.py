"""ctypes binding of include/pacmap.h (libpacmap_b200.so). No fallback: a missing library is an error."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_PKG), "lib", "libpacmap_b200.so")

PACMAP_OK = 0


class Config(C.Structure):
    """struct pacmap_config (include/pacmap.h)."""

    _fields_ = [
        ("embedding_dimensions", C.c_uint64),
        ("init_kind", C.c_int32),
        ("init_value", C.c_void_p),
        ("init_has_seed", C.c_int32),
        ("init_seed", C.c_uint64),
        ("mid_near_ratio", C.c_float),
        ("far_pair_ratio", C.c_float),
        ("has_override_neighbors", C.c_int32),
        ("override_neighbors", C.c_uint64),
        ("has_seed", C.c_int32),
        ("seed", C.c_uint64),
        ("pair_kind", C.c_int32),
        ("pair_neighbors", C.c_void_p),
        ("pair_neighbors_rows", C.c_uint64),
        ("pair_mn", C.c_void_p),
        ("pair_mn_rows", C.c_uint64),
        ("pair_fp", C.c_void_p),
        ("pair_fp_rows", C.c_uint64),
        ("learning_rate", C.c_float),
        ("num_iters", C.c_uint64 * 3),
        ("snapshots", C.c_void_p),
        ("n_snapshots", C.c_uint64),
        ("approx_threshold", C.c_uint64),
        ("knn_mode", C.c_int32),
        ("device", C.c_int32),
        ("loss_trace", C.c_void_p),
        ("metric", C.c_int32),
    ]


_lib = None

_vp, _u64, _i32, _f32 = C.c_void_p, C.c_uint64, C.c_int32, C.c_float
_SIGS = {
    "pacmap_config_default": (Config, []),
    "pacmap_fit_transform": (C.c_int, [_vp, _u64, _u64, C.POINTER(Config), _vp, _vp]),
    "pacmap_fit_transform_device": (C.c_int, [_vp, _u64, _u64, C.POINTER(Config), _vp, _vp]),
    "pacmap_knn_exact": (C.c_int, [_vp, _u64, _u64, _u64, _i32, _i32, _vp, _vp]),
    "pacmap_knn_exact_shard": (C.c_int, [_vp, _u64, _u64, _u64, _i32, C.c_uint32, C.c_uint32, _i32, _vp, _vp, _vp]),
    "pacmap_preprocess": (C.c_int, [_vp, _u64, _u64, _i32, _vp, _vp, _vp, _vp]),
    "pacmap_generate_pairs": (C.c_int, [_vp, _u64, _u64, C.POINTER(Config), _vp, _vp, _vp, _vp]),
    "pacmap_reselect_neighbors": (C.c_int, [_vp, _vp, _u64, _u64, _u64, _i32, _vp, _vp]),
    "pacmap_sample_pairs": (C.c_int, [_vp, _u64, _u64, _vp, _u64, _u64, _u64, _u64, _i32, _vp, _vp]),
    "pacmap_optimize_steps": (C.c_int, [_vp, _vp, _vp, _u64, _u64, _vp, _u64, _vp, _u64, _vp, _u64, _f32, _u64,
                                        _u64, _u64, _u64, _i32, _vp]),
    "pacmap_gradient": (C.c_int, [_vp, _u64, _u64, _vp, _u64, _vp, _u64, _vp, _u64, _f32, _f32, _f32, _i32, _vp]),
    "pacmap_init_value": (C.c_int, [_vp, _u64, _u64, _i32, _vp]),
    "pacmap_init_random": (C.c_int, [_u64, _u64, _u64, _i32, _vp]),
    "pacmap_quality": (C.c_int, [_vp, _u64, _u64, _vp, _u64, _vp, _u64, _u64, _vp, _u64, _i32, _vp, _vp]),
    "pacmap_mlp_param_count": (C.c_uint64, [_u64, _u64]),
    "pacmap_mlp_init": (C.c_int, [_u64, _u64, _u64, _vp]),
    "pacmap_mlp_train": (C.c_int, [_vp, _vp, _u64, _u64, _u64, _u64, _u64, _f32, _f32, _u64, _i32, _vp, _vp]),
    "pacmap_mlp_apply": (C.c_int, [_vp, _u64, _u64, _vp, _u64, _i32, _vp]),
    "pacmap_mlp_grad": (C.c_int, [_vp, _u64, _u64, _vp, _vp, _u64, _i32, _vp, _vp]),
    "pacmap_fit_transform_learned": (C.c_int, [_vp, _u64, _u64, C.POINTER(Config), _vp, _vp, _vp, _vp, _vp]),
    "pacmap_fit_transform_learned_device": (C.c_int, [_vp, _u64, _u64, C.POINTER(Config), _vp, _vp, _vp, _vp,
                                                      _vp]),
    "pacmap_pca_axes": (C.c_int, [_vp, _u64, _u64, _vp]),
    "pacmap_model_target_stats": (C.c_int, [_vp, _u64, _u64, _vp, _vp]),
    "pacmap_model_save": (C.c_int, [C.c_char_p, _u64, _u64, _vp, _f32, _f32, _vp, _vp, _vp]),
    "pacmap_model_load": (C.c_int, [C.c_char_p, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "pacmap_transform": (C.c_int, [_vp, _u64, _u64, _u64, _vp, _f32, _f32, _vp, _vp, _vp, _i32, _vp]),
    "pacmap_device_stream": (C.c_void_p, [_i32]),
    "pacmap_take_launch_count": (C.c_uint64, []),
    "pacmap_gather_rate": (C.c_int, [_i32, C.c_void_p]),
    "pacmap_knn_exact_shard_device": (C.c_int, [_vp, _u64, _u64, _u64, _i32, C.c_uint32, C.c_uint32, _i32, _vp, _vp,
                                                _vp]),
    "pacmap_debug_stall_knn_loads": (C.c_int, [_i32, _i32]),
    "pacmap_set_stage_timing": (None, [_i32]),
    "pacmap_stage_times": (C.c_uint64, [_vp, _u64]),
    "pacmap_last_error": (C.c_char_p, []),
    "pacmap_version": (C.c_char_p, []),
}


def lib():
    """Load libpacmap_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python pacmap-rs_b200/build.py`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def ptr(a):
    """Raw pointer of a C-contiguous numpy array (or None)."""
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.flags["C_CONTIGUOUS"], "expected a C-contiguous numpy array"
    return C.c_void_p(a.ctypes.data)


def last_error() -> str:
    return lib().pacmap_last_error().decode()
