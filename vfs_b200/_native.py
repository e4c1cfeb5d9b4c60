"""Loader of the in-tree CUDA library (vfs_b200/_lib/libvfs_b200.so) and its ctypes signatures.

There is no fallback: if the library is missing or cannot be loaded, importing the solver
raises, so nothing silently runs without the CUDA kernels.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libvfs_b200.so")

VFS_OK = 0
STATUS = {
    -1: "invalid argument", -2: "CUDA error", -3: "invalid call order", -4: "out of device memory",
    -5: "file error", -6: "device wait timed out", -7: "not enough free device memory",
}


class VfsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, 'error')} ({status}): {message}")
        self.status = status


_lib = None

_vp = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float
_sz = ctypes.c_size_t

# name -> argtypes (all return int unless listed in _RESTYPE)
SIGNATURES = {
    "vfs_status_string": [_i],
    "vfs_last_error": [_vp],
    "vfs_version": [],
    "vfs_create": [ctypes.POINTER(_vp)],
    "vfs_create_ex": [ctypes.POINTER(_vp), _i, _i, _i],
    "vfs_destroy": [_vp],
    "vfs_set_stream": [_vp, _vp],
    "vfs_synchronize": [_vp],
    "vfs_initialize": [_vp, _i, _i, _f, _f, _f, _f, _f, _f, _i, _f, _i, _i],
    "vfs_set_limit_range": [_vp, _f],
    "vfs_set_camera": [_vp, _f, _f],
    "vfs_set_tensor_math": [_vp, _i],
    "vfs_set_warm_start": [_vp, _i],
    "vfs_cached_graphs": [_vp],
    "vfs_batch_cached_graphs": [_vp],
    "vfs_tuning_solves": [],
    "vfs_state_bytes": [_vp],
    "vfs_export_state": [_vp, _vp, _sz],
    "vfs_import_state": [_vp, _vp, _sz],
    "vfs_debug_fail_allocation": [_i],
    "vfs_debug_check_guards": [_vp, ctypes.POINTER(ctypes.c_int)],
    "vfs_get_level_size": [_vp, _i, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i)],
    "vfs_load_vector_fields": [_vp, _vp, _vp],
    "vfs_copy_mask_to_device": [_vp, _vp],
    "vfs_copy_images_to_device_u8": [_vp, _vp, _vp],
    "vfs_copy_images_to_device_f32": [_vp, _vp, _vp],
    "vfs_copy_images_to_device_u8c3": [_vp, _vp, _vp],
    "vfs_copy_images_from_device_u8": [_vp, _vp, _vp],
    "vfs_solve_stereo_forward": [_vp],
    "vfs_solve_stereo_forward_masked": [_vp],
    "vfs_copy_1d_disparity_to_host": [_vp, _vp],
    "vfs_copy_disparity_to_host": [_vp, _vp],
    "vfs_copy_warped_image_to_host": [_vp, _vp],
    "vfs_copy_1d_disparity_to_device": [_vp, _vp],
    "vfs_copy_disparity_to_device": [_vp, _vp],
    "vfs_copy_stereo_to_host": [_vp, _vp, _vp] + [_f] * 11,
    "vfs_copy_disparity_vis_to_host": [_vp, _vp, _f],
    "vfs_debug_get_buffer": [_vp, ctypes.c_char_p, _i, _vp],
    "vfs_set_solve_path": [_vp, _i, _i],
    "vfs_set_graph": [_vp, _i],
    "vfs_batch_create": [ctypes.POINTER(_vp)],
    "vfs_batch_destroy": [_vp],
    "vfs_batch_last_error": [_vp],
    "vfs_batch_set_stream": [_vp, _vp],
    "vfs_batch_add": [_vp, _vp],
    "vfs_batch_clear": [_vp],
    "vfs_batch_size": [_vp],
    "vfs_batch_set_storage": [_vp, _i],
    "vfs_batch_set_graph": [_vp, _i],
    "vfs_batch_solve": [_vp, _i],
    "vfs_batch_solve_host": [_vp, _vp, _vp, _vp, _i],
    "vfs_batch_solve_device": [_vp, _vp, _vp, _vp, _i],
    "vfs_batch_set_autotune": [_vp, _i],
    "vfs_batch_set_mode": [_vp, _i],
    "vfs_batch_set_fine_concurrency": [_vp, _i],
    "vfs_batch_set_pipeline": [_vp, _i, _i],
    "vfs_set_autotune": [_vp, _i],
    "vfs_set_iteration_variant": [_vp, _i],
    "vfs_get_iteration_variants": [_vp, _vp, _i, ctypes.POINTER(_i)],
    "vfs_set_iteration_variants": [_vp, _vp, _i],
    "vfs_batch_set_iteration_variants": [_vp, _vp, _i],
    "vfs_batch_set_iteration_variant": [_vp, _i],
    "vfs_equalize_hist_u8": [_vp, _vp, _sz, _vp],
    "vfs_equalize_hist_u8_noalloc": [_vp, _vp, _sz, _i, _vp],
    "vfs_estimate_device_bytes": [_i, _i, _i, _f, _i, _i],
    "vfs_launch_count": [],
    "vfs_device_status": [_vp],
    "vfs_set_launch_overlap": [_i],
    "vfs_profile_enable": [_vp, _i],
    "vfs_profile_reset": [_vp],
    "vfs_profile_read": [_vp, _i, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_double),
                         ctypes.POINTER(ctypes.c_double)],
    "vfs_profile_epoch": [_vp],
    "vfs_profile_intervals": [_vp, _i, _i, _vp, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_int)],
    "Create": [],
    "Init": [_vp, _i, _i, _f, _f, _f, _f, _f, _f, _i, _f, _i, _i, _f, _f, ctypes.c_char_p, ctypes.c_char_p,
             ctypes.c_char_p],
    "SolveStereo": [_vp, _vp, _vp, _vp, _i, _i, _f],
}
_RESTYPE = {
    "vfs_estimate_device_bytes": ctypes.c_size_t,
    "vfs_launch_count": ctypes.c_longlong,
    "vfs_tuning_solves": ctypes.c_longlong,
    "vfs_state_bytes": ctypes.c_size_t,
    "vfs_status_string": ctypes.c_char_p,
    "vfs_last_error": ctypes.c_char_p,
    "vfs_batch_last_error": ctypes.c_char_p,
    "Create": _vp,
    "Init": None,
    "SolveStereo": None,
}


def lib():
    """Load the CUDA library (raises if it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"vfs_b200 CUDA library not built: {LIB_PATH} is missing "
                              "(run `python -m vfs_b200.build`)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, _i)
        _lib = L
    return _lib


def check(handle, status: int) -> None:
    if status != VFS_OK:
        msg = lib().vfs_last_error(handle) or b""
        raise VfsError(status, msg.decode(errors="replace"))


def check_batch(handle, status: int) -> None:
    if status != VFS_OK:
        msg = lib().vfs_batch_last_error(handle) or b""
        raise VfsError(status, msg.decode(errors="replace"))
