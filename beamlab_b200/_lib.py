"""Loads the in-tree CUDA library (beamlab_b200/_build/libbeamlab_b200.so) and declares the C ABI's signatures.

The library is required: if it is missing, importing the World fails loudly (build it with
``python -m beamlab_b200.build`` or ``__graft_entry__.build()``); nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libbeamlab_b200.so")
HEADER = os.path.join(HERE, "..", "include", "beamlab_gpu.h")

_lib = None

_vp, _i32, _f = C.c_void_p, C.c_int32, C.c_float
_SIGNATURES = {
    "bl_gpu_default_config": ([_vp], None),
    "bl_gpu_create": ([_vp, _vp], C.c_int),
    "bl_gpu_destroy": ([_vp], C.c_int),
    "bl_gpu_set_terrain": ([_vp, _i32, _i32, _f, _f, _f, _vp, _vp], C.c_int),
    "bl_gpu_add_box": ([_vp, _vp, _vp, _vp, _i32, _f], C.c_int),
    "bl_gpu_add_cylinder": ([_vp, _vp, _f, _f, _i32], C.c_int),
    "bl_gpu_build_grid": ([_vp], C.c_int),
    "bl_gpu_set_kill_y": ([_vp, _f], C.c_int),
    "bl_gpu_add_body": ([_vp, _vp, _vp], C.c_int),
    "bl_gpu_step_substeps": ([_vp, _i32, _vp], C.c_int),
    "bl_gpu_download_nodes": ([_vp, _i32, _vp], C.c_int),
    "bl_gpu_upload_nodes": ([_vp, _i32, _vp], C.c_int),
    "bl_gpu_download_beams": ([_vp, _i32, _vp], C.c_int),
    "bl_gpu_body_state": ([_vp, _i32, _vp], C.c_int),
    "bl_gpu_stats": ([_vp, _vp], C.c_int),
    "bl_gpu_synchronize": ([_vp], C.c_int),
    "bl_gpu_device_nodes": ([_vp, _vp, _vp], C.c_int),
    "bl_gpu_upload_all_nodes": ([_vp, _vp, _i32, _vp], C.c_int),
    "bl_gpu_download_all_nodes": ([_vp, _vp, _i32, _vp], C.c_int),
    "bl_gpu_profile_frame": ([_vp, _i32, _vp, _vp], C.c_int),
    "bl_gpu_body_range": ([_vp, _i32, _vp, _vp, _vp, _vp], C.c_int),
    "bl_gpu_substep_noalloc": ([_vp, _i32, _vp, _i32, _vp, _vp, _vp, _f, _i32, _i32, _i32, _vp], C.c_int),
    "bl_gpu_set_node_force": ([_vp, _i32, _i32, _vp], C.c_int),
    "bl_gpu_set_wheel_drive": ([_vp, _i32, _i32, _f, _f], C.c_int),
    "bl_gpu_download_wheels": ([_vp, _i32, _vp, _vp, _vp], C.c_int),
    "bl_gpu_wheel_speed": ([_vp, _i32, _vp, _vp], C.c_int),
    "bl_gpu_download_fem": ([_vp, _i32, _vp, _vp, _vp, _vp, _vp], C.c_int),
    "bl_gpu_download_fem_tris": ([_vp, _i32, _vp, _vp, _vp, _vp], C.c_int),
    "bl_gpu_download_pairs": ([_vp, _vp, _i32, _vp], C.c_int),
    "bl_gpu_fem_stats": ([_vp, _vp], C.c_int),
    "bl_gpu_mlp_init": ([_vp, C.c_uint64], C.c_int),
    "bl_gpu_mlp_set_weights": ([_vp, _vp, _i32], C.c_int),
    "bl_gpu_mlp_get_weights": ([_vp, _vp, _i32], C.c_int),
    "bl_gpu_mlp_record": ([_vp, _i32], C.c_int),
    "bl_gpu_mlp_samples": ([_vp, _vp], C.c_int),
    "bl_gpu_mlp_train": ([_vp, _i32, _i32, _f, C.c_uint64, _vp], C.c_int),
    "bl_gpu_mlp_forward": ([_vp, _vp, _i32, _vp], C.c_int),
    "bl_gpu_mlp_gradient": ([_vp, _vp, _vp, _vp, _i32, _vp, _vp], C.c_int),
    "bl_fem_pattern": ([_vp, _vp, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
    "bl_gpu_error_string": ([C.c_int], C.c_char_p),
    "bl_gpu_last_cuda_error": ([_vp], C.c_int),
    "bl_gpu_abi_version": ([], C.c_int),
}


def header_symbols(path: str = HEADER) -> list[str]:
    """The function names include/beamlab_gpu.h declares."""
    text = open(path).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(bl_gpu_\w+)\s*\(", text, re.M)))


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"beamlab_b200: CUDA library not built ({LIB_PATH}); run `python -m beamlab_b200.build`")
    L = C.CDLL(LIB_PATH)
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L
