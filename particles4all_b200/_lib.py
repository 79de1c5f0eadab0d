"""Loads the in-tree libp4a.so (CUDA sm_100a kernels behind the C ABI of
include/p4a.h) and declares its signatures. There is no fallback: if the library
is missing or no usable GPU is present, the calls that need the device fail."""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libp4a.so")

# Every entry point declared in include/p4a.h, with its ctypes signature.
_vp, _i32, _dbl, _sz, _f32 = C.c_void_p, C.c_int32, C.c_double, C.c_size_t, C.c_float
SIGNATURES = {
    "p4a_abi_version": ([], C.c_int),
    "p4a_status_string": ([C.c_int], C.c_char_p),
    "p4a_default_params": ([C.c_char_p, _vp], C.c_int),
    "p4a_device_check": ([C.c_int], C.c_int),
    "p4a_create": ([C.c_int, C.POINTER(_vp)], C.c_int),
    "p4a_destroy": ([_vp], C.c_int),
    "p4a_last_error": ([_vp], C.c_char_p),
    "p4a_set_stream": ([_vp, _vp], C.c_int),
    "p4a_synchronize": ([_vp], C.c_int),
    "p4a_reset": ([_vp, _vp], C.c_int),
    "p4a_reset_scene": ([_vp, _vp, _vp], C.c_int),
    "p4a_step": ([_vp, _dbl, C.POINTER(_i32)], C.c_int),
    "p4a_append_fluid": ([_vp, _vp, _vp, _i32, C.POINTER(_i32)], C.c_int),
    "p4a_apply_ray_impulse": ([_vp, _vp, _vp, _vp, _dbl, _dbl], C.c_int),
    "p4a_hold_body": ([_vp, _i32, _vp, _dbl, _dbl], C.c_int),
    "p4a_release_body": ([_vp], C.c_int),
    "p4a_resize_box": ([_vp, _vp], C.c_int),
    "p4a_get_info": ([_vp, _vp], C.c_int),
    "p4a_buffer": ([_vp, _i32, _i32, C.POINTER(_vp), C.POINTER(_sz)], C.c_int),
    "p4a_read": ([_vp, _i32, _i32, _vp, _sz, _sz], C.c_int),
    "p4a_write": ([_vp, _i32, _i32, _vp, _sz, _sz], C.c_int),
    "p4a_read_async": ([_vp, _i32, _i32, _vp, _sz, _sz], C.c_int),
    "p4a_read_wait": ([_vp], C.c_int),
    "p4a_get_stats": ([_vp, _i32, _vp], C.c_int),
    "p4a_body_pose": ([_vp, _i32, _vp, _vp, _i32], C.c_int),
    "p4a_aniso": ([_vp, _vp], C.c_int),
    "p4a_default_aniso_params": ([_vp], C.c_int),
    "p4a_grid_sort_workspace_size": ([_i32, _i32], _sz),
    "p4a_grid_sort": ([_vp, _i32, _f32, _f32] + [_vp] * 11 + [_vp, _sz, _vp, _vp], C.c_int),
    "p4a_test_scan_wait": ([C.c_uint32, _i32], C.c_int),
    "p4a_hose_emit": ([_vp, _vp, C.c_int64, C.POINTER(_i32)], C.c_int),
    "p4a_build_scene": ([_vp] * 8, C.c_int),
    "p4a_profile_enable": ([_vp, _i32], C.c_int),
    "p4a_profile_reset": ([_vp], C.c_int),
    "p4a_profile_read": ([_vp, _vp, _i32, C.POINTER(_i32)], C.c_int),
    "p4a_kernel_launches": ([], C.c_uint64),
    "p4a_grid_sort_noalloc": ([_vp, _i32, _f32, _f32] + [_vp] * 11 + [_vp, _vp], C.c_int),
    "p4a_batch_create": ([C.c_int, _vp, C.POINTER(_vp)], C.c_int),
    "p4a_batch_footprint": ([_vp, C.POINTER(C.c_int64)], C.c_int),
    "p4a_batch_destroy": ([_vp], C.c_int),
    "p4a_batch_last_error": ([_vp], C.c_char_p),
    "p4a_batch_set_stream": ([_vp, _vp], C.c_int),
    "p4a_batch_add_scene": ([_vp, _vp, _vp, C.POINTER(_i32)], C.c_int),
    "p4a_batch_add_preset": ([_vp, _vp, C.POINTER(_i32)], C.c_int),
    "p4a_batch_remove_scene": ([_vp, _i32], C.c_int),
    "p4a_batch_step": ([_vp, _vp, _i32, _dbl], C.c_int),
    "p4a_batch_synchronize": ([_vp], C.c_int),
    "p4a_batch_usage_get": ([_vp, _vp], C.c_int),
    "p4a_batch_scene_info": ([_vp, _i32, _vp], C.c_int),
    "p4a_batch_read": ([_vp, _i32, _i32, _i32, _vp, _sz, _sz], C.c_int),
    "p4a_batch_write": ([_vp, _i32, _i32, _i32, _vp, _sz, _sz], C.c_int),
    "p4a_batch_stats": ([_vp, _i32, _vp], C.c_int),
    "p4a_batch_use_graphs": ([_vp, _i32], C.c_int),
    "p4a_batch_read_async": ([_vp, _i32, _i32, _i32, _vp, _sz, _sz], C.c_int),
    "p4a_batch_write_async": ([_vp, _i32, _i32, _i32, _vp, _sz, _sz], C.c_int),
    "p4a_batch_step_io": ([_vp, _vp, _i32, C.c_double, _i32], C.c_int),
    "p4a_batch_set_lanes": ([_vp, _i32, C.c_int64], C.c_int),
    "p4a_batch_profile_enable": ([_vp, _i32], C.c_int),
    "p4a_batch_profile_reset": ([_vp], C.c_int),
    "p4a_batch_profile_read": ([_vp, _vp, _i32, C.POINTER(_i32)], C.c_int),
    "p4a_server_default_config": ([_vp], C.c_int),
    "p4a_server_create": ([C.c_int, _vp, C.POINTER(_vp)], C.c_int),
    "p4a_server_destroy": ([_vp], C.c_int),
    "p4a_server_last_error": ([_vp], C.c_char_p),
    "p4a_server_clock": ([_vp], _dbl),
    "p4a_server_create_scene": ([_vp, _vp, _vp, C.POINTER(_i32), C.POINTER(C.c_int64)], C.c_int),
    "p4a_server_step": ([_vp, _i32, _dbl, _vp, _vp, _sz, C.POINTER(C.c_int64)], C.c_int),
    "p4a_server_destroy_scene": ([_vp, _i32, C.POINTER(C.c_int64)], C.c_int),
    "p4a_server_poll": ([_vp, _vp, _i32, C.POINTER(_i32), _dbl], C.c_int),
    "p4a_server_get_stats": ([_vp, _vp], C.c_int),
    "p4a_kernel_shapes": ([_i32, _vp, _vp, _i32, C.POINTER(_i32)], C.c_int),
    "p4a_tune_set": ([_i32, C.c_int64, _i32], C.c_int),
    "p4a_tune_clear": ([_i32], C.c_int),
    "p4a_tune_get": ([_i32, C.c_int64, C.POINTER(_i32)], C.c_int),
    "p4a_default_mesh_params": ([_vp], C.c_int),
    "p4a_mesh": ([_vp, _vp, C.POINTER(C.c_int64)], C.c_int),
    "p4a_mesh_get_info": ([_vp, _vp], C.c_int),
    "p4a_default_ssfr_params": ([_vp], C.c_int),
    "p4a_ssfr": ([_vp, _vp, _vp, _i32], C.c_int),
    "p4a_ssfr_get_info": ([_vp, _vp], C.c_int),
    "p4a_ssfr_buffer": ([_vp, _i32, C.POINTER(_vp), C.POINTER(_sz)], C.c_int),
    "p4a_ssfr_read": ([_vp, _i32, _vp, _sz], C.c_int),
    "p4a_default_ray_params": ([_vp], C.c_int),
    "p4a_ray": ([_vp, _vp, _vp, _i32], C.c_int),
    "p4a_ray_buffer": ([_vp, C.POINTER(_vp), C.POINTER(_sz), C.POINTER(_i32), C.POINTER(_i32)], C.c_int),
    "p4a_ray_read": ([_vp, _vp, _sz], C.c_int),
    "p4a_set_environment": ([_vp, _vp, _i32, _i32], C.c_int),
    "p4a_environment_read": ([_vp, C.POINTER(_i32), _vp, _sz], C.c_int),
}

_lib = None


class P4AError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"p4a status {status}: {message}")
        self.status = status


def lib():
    """The loaded libp4a.so. Raises if it has not been built (no silent fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise P4AError(7, f"{LIB_PATH} is missing: build it with particles4all_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
        from . import autotune
        autotune.load(L=L)  # measured launch shapes, when tuning.json is present
    return _lib


def check(rc, handle=None, what=""):
    if rc != 0:
        L = lib()
        msg = L.p4a_last_error(handle).decode() if handle else L.p4a_status_string(rc).decode()
        raise P4AError(rc, f"{what}: {msg}" if what else msg)
    return rc


def device_available(device=0):
    """True when libp4a loads and `device` is a B200-class (sm_100) GPU."""
    try:
        return lib().p4a_device_check(device) == 0
    except (OSError, P4AError):
        return False
