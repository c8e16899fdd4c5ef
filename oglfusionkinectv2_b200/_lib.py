"""ctypes binding of libkf.so (the C ABI in include/kf.h).

The library is loaded from this package directory only; if it is missing the import
fails loudly (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libkf.so")

KF_OK = 0
KF_ERR_INVALID_ARGUMENT = -1
KF_ERR_OUT_OF_MEMORY = -2
KF_ERR_CUDA = -3
KF_ERR_NO_DEVICE = -4
KF_ERR_TIMEOUT = -5
KF_ERR_STATE = -6
KF_ERR_IO = -7
KF_ERR_CAPACITY = -8
KF_ERR_ADMISSION = -9

KF_STORAGE_F32F32 = 0
KF_STORAGE_F16U16 = 1
KF_STORAGE_RG16I = 2
KF_JTJ_FP32 = 0
KF_JTJ_SPLIT_BF16 = 1
KF_TRACK_ICP = 0
KF_TRACK_SDF = 1
KF_MC_HISTOPYRAMID = 0
KF_MC_SCAN = 1
KF_BATCH_MAX_SESSIONS = 255

KF_Q1_LAST_GROUP_ONLY = 1 << 0
KF_Q3_DOWN_FROM_LEFT = 1 << 1
KF_Q6_SDF_D2_TWICE = 1 << 2
KF_Q7_SDF_LAST_COLUMN = 1 << 3
KF_Q13_MC_FIRST_SEVEN = 1 << 4
KF_Q15_MC_BORDER_SKIP = 1 << 5
KF_Q18_STL_COUNT_X4 = 1 << 6
KF_Q23_SDF_XY_OFFSET = 1 << 7
KF_Q19_EIG_TRANSLATION = 1 << 8
KF_Q24_MC_SHADER_UNITS = 1 << 11
KF_Q8_NARROW_BAND = 1 << 9
KF_Q4_SAME_PIXEL = 1 << 10
KF_QUIRKS_REFERENCE = (KF_Q1_LAST_GROUP_ONLY | KF_Q3_DOWN_FROM_LEFT | KF_Q4_SAME_PIXEL
                       | KF_Q6_SDF_D2_TWICE | KF_Q7_SDF_LAST_COLUMN | KF_Q8_NARROW_BAND
                       | KF_Q13_MC_FIRST_SEVEN | KF_Q15_MC_BORDER_SKIP | KF_Q19_EIG_TRANSLATION
                       | KF_Q23_SDF_XY_OFFSET)
KF_QUIRKS_DEFAULT = KF_QUIRKS_REFERENCE & ~KF_Q1_LAST_GROUP_ONLY
KF_QUIRKS_TRACKING = KF_QUIRKS_DEFAULT & ~(KF_Q4_SAME_PIXEL | KF_Q8_NARROW_BAND)


class kf_config(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("dim_x", C.c_float), ("dim_y", C.c_float), ("dim_z", C.c_float),
                ("mu", C.c_float), ("max_weight", C.c_float),
                ("near_plane", C.c_float), ("far_plane", C.c_float),
                ("dist_threshold", C.c_float), ("normal_threshold", C.c_float),
                ("iterations", C.c_int32 * 3), ("storage", C.c_int32), ("jtj", C.c_int32),
                ("tracking", C.c_int32), ("quirks", C.c_uint32),
                ("integrate_every", C.c_int32), ("reserved", C.c_int32 * 7)]


class kf_intrinsics(C.Structure):
    _fields_ = [("fx", C.c_float), ("fy", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
                ("width", C.c_int32), ("height", C.c_int32)]


class kf_volume_view(C.Structure):
    _fields_ = [("device_ptr", C.c_void_p), ("nx", C.c_int32), ("ny", C.c_int32),
                ("nz", C.c_int32), ("storage", C.c_int32), ("value_bytes", C.c_int64),
                ("weight_offset_bytes", C.c_int64), ("row_pitch_bytes", C.c_int64),
                ("slice_pitch_bytes", C.c_int64)]


class kf_launch_shape(C.Structure):
    _fields_ = [("integrate_z_chunk", C.c_int32), ("raycast_rows", C.c_int32), ("reserved", C.c_int32 * 6)]


class kf_ir_camera(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("fx", "fy", "cx", "cy", "k1", "k2", "k3", "p1", "p2")]


class KfError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what}: {status_string(status)} ({status})")
        self.status = status


_P = C.c_void_p
_I = C.c_int
_PD = C.POINTER(C.c_double)
_PF = C.POINTER(C.c_float)

# name: (restype, argtypes)
SIGNATURES = {
    "kf_abi_version": (_I, []),
    "kf_status_string": (C.c_char_p, [_I]),
    "kf_config_default": (_I, [C.POINTER(kf_config)]),
    "kf_create": (_I, [C.POINTER(kf_config), C.POINTER(kf_intrinsics), C.POINTER(_P)]),
    "kf_destroy": (_I, [_P]),
    "kf_last_error": (C.c_char_p, [_P]),
    "kf_session_device_bytes": (_I, [C.POINTER(kf_config), C.POINTER(kf_intrinsics),
                                     C.POINTER(C.c_uint64)]),
    "kf_reset": (_I, [_P, _PD, _I]),
    "kf_reset_volume": (_I, [_P]),
    "kf_reset_pose": (_I, [_P, _PD]),
    "kf_set_pose": (_I, [_P, _PD]),
    "kf_get_pose": (_I, [_P, _PD]),
    "kf_set_config": (_I, [_P, C.POINTER(kf_config)]),
    "kf_depth_to_vertex_f32": (_I, [_P, _P]),
    "kf_depth_to_vertex_u16": (_I, [_P, _P]),
    "kf_depth_to_vertex_u16_device": (_I, [_P, _P]),
    "kf_vertex_to_normal": (_I, [_P]),
    "kf_track_icp": (_I, [_P, C.POINTER(_I)]),
    "kf_track_sdf": (_I, [_P, C.POINTER(_I)]),
    "kf_recover_pose": (_I, [_P, C.POINTER(_I)]),
    "kf_get_alignment_energy": (_I, [_P, _PF]),
    "kf_get_reduction": (_I, [_P, _PF]),
    "kf_get_iterations_run": (_I, [_P, C.POINTER(_I)]),
    "kf_integrate": (_I, [_P]),
    "kf_raycast": (_I, [_P]),
    "kf_frame_step_u16": (_I, [_P, _P, C.POINTER(_I)]),
    "kf_frame_step_u16_device": (_I, [_P, _P, C.POINTER(_I)]),
    "kf_get_raycast": (_I, [_P, _P, _P]),
    "kf_set_reference_maps": (_I, [_P, _P, _P]),
    "kf_get_vertex_map": (_I, [_P, _I, _P]),
    "kf_get_normal_map": (_I, [_P, _I, _P]),
    "kf_get_depth_map": (_I, [_P, _I, _P]),
    "kf_get_track_status": (_I, [_P, _I, _P]),
    "kf_get_volume": (_I, [_P, C.POINTER(kf_volume_view)]),
    "kf_copy_volume_to_host": (_I, [_P, _P, C.c_uint64]),
    "kf_copy_volume_from_host": (_I, [_P, _P, C.c_uint64]),
    "kf_get_cum_twist": (_I, [_P, _PD]),
    "kf_intensity_projection": (_I, [_P, _P]),
    "kf_frame_step_u16_async": (_I, [_P, _P]),
    "kf_frame_sync": (_I, [_P, C.POINTER(_I)]),
    "kf_get_last_result": (_I, [_P, _PD, C.POINTER(_I)]),
    "kf_set_depth_undistortion": (_I, [_P, C.POINTER(kf_ir_camera)]),
    "kf_get_undistortion_map": (_I, [_P, _P]),
    "kf_set_depth_filter": (_I, [_P, _I]),
    "kf_set_launch_shape": (_I, [_P, C.POINTER(kf_launch_shape)]),
    "kf_get_launch_shape": (_I, [_P, C.POINTER(kf_launch_shape)]),
    "kf_autotune": (_I, [_P, _I, C.POINTER(kf_launch_shape), _PF]),
    "kf_batch_frame_step_u16_device_async": (_I, [_P, _P, _P, _I]),
    "kf_batch_sync": (_I, [_P]),
    "kf_batch_get_tracked": (_I, [_P, _I, _P]),
    "kf_batch_set_launch_shape": (_I, [_P, C.POINTER(kf_launch_shape)]),
    "kf_batch_get_launch_shape": (_I, [_P, C.POINTER(kf_launch_shape)]),
    "kf_batch_autotune": (_I, [_P, _P, _I, _I, C.POINTER(kf_launch_shape), _PF]),
    "kf_save_volume": (_I, [_P, C.c_char_p]),
    "kf_load_volume": (_I, [_P, C.c_char_p]),
    "kf_selftest_barrier_timeout": (_I, [_P, C.c_longlong]),
    "kf_get_pose_library_size": (_I, [_P, C.POINTER(_I)]),
    "kf_get_stage_times": (_I, [_P, _PF]),
    "kf_get_stage_stats": (_I, [_P, _PD, C.POINTER(C.c_uint64)]),
    "kf_reset_stage_stats": (_I, [_P]),
    "kf_set_stage_timing": (_I, [_P, _I]),
    "kf_get_stage_timing": (_I, [_P, C.POINTER(C.c_int)]),
    "kf_get_launch_count": (_I, [_P, C.POINTER(C.c_uint64)]),
    "kf_get_stream": (_I, [_P, C.POINTER(_P)]),
    "kf_mc_extract": (_I, [_P, C.c_float, _I, C.POINTER(C.c_uint32)]),
    "kf_mc_copy_vertices": (_I, [_P, _P, C.c_uint64]),
    "kf_mc_copy_base_level": (_I, [_P, _P, C.c_uint64]),
    "kf_mc_export_stl": (_I, [_P, C.c_char_p]),
    "kf_mc_export_ply": (_I, [_P, C.c_char_p]),
    "kf_mc_copy_normals": (_I, [_P, _P, C.c_uint64]),
    "kf_mc_extract_mesh": (_I, [_P, C.c_float, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "kf_mc_copy_mesh": (_I, [_P, _P, _P, _P, C.c_uint64, C.c_uint64]),
    "kf_mc_export_mesh_ply": (_I, [_P, C.c_char_p]),
    "kf_mc_export_mesh_stl": (_I, [_P, C.c_char_p]),
    "kf_prefix_sum_u32": (_I, [_P, _P, C.c_uint64, C.POINTER(C.c_uint32), _P]),
    "kf_prefix_sum_u32_noalloc": (_I, [_P, _P, C.c_uint64, C.POINTER(C.c_uint32), _P]),
    "kf_batch_create": (_I, [_I, C.POINTER(_P)]),
    "kf_batch_destroy": (_I, [_P]),
    "kf_batch_last_error": (C.c_char_p, [_P]),
    "kf_batch_frame_step_u16": (_I, [_P, C.POINTER(_P), C.POINTER(_P), _I, C.POINTER(C.c_int32)]),
    "kf_batch_frame_step_u16_device": (_I, [_P, C.POINTER(_P), C.POINTER(_P), _I, C.POINTER(C.c_int32)]),
    "kf_batch_get_stage_times": (_I, [_P, C.POINTER(C.c_float)]),
    "kf_batch_get_poses": (_I, [_P, _I, _P]),
    "kf_batch_get_launch_count": (_I, [_P, C.POINTER(C.c_uint64)]),
    "kf_server_config_default": (_I, [_P]),
    "kf_server_create": (_I, [_P, C.POINTER(_P)]),
    "kf_server_destroy": (_I, [_P]),
    "kf_server_last_error": (C.c_char_p, [_P]),
    "kf_server_now": (C.c_double, []),
    "kf_server_open": (_I, [_P, _P, _P, _P, C.POINTER(_I)]),
    "kf_server_close": (_I, [_P, _I]),
    "kf_server_prewarm": (_I, [_P, _P, _P, _I, C.POINTER(_I)]),
    "kf_server_submit": (_I, [_P, _I, _P]),
    "kf_server_submit_device": (_I, [_P, _I, _P]),
    "kf_server_step": (_I, [_P, C.POINTER(_I)]),
    "kf_server_step_async": (_I, [_P, C.POINTER(_I)]),
    "kf_server_sync": (_I, [_P, C.POINTER(_I)]),
    "kf_server_get_pose": (_I, [_P, _I, _P, C.POINTER(_I), C.POINTER(C.c_uint64)]),
    "kf_server_pending": (_I, [_P, _I, C.POINTER(_I)]),
    "kf_server_last_step": (_I, [_P, _I, _P, _P, _P, C.POINTER(_I)]),
    "kf_server_stats": (_I, [_P, _P]),
    "kf_server_reset_stats": (_I, [_P]),
}

_lib = None


class ServerConfig(C.Structure):
    """kf_server_config (kf.h)."""
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_sessions", C.c_int32), ("max_batch", C.c_int32),
                ("storage", C.c_int32), ("jtj", C.c_int32), ("reserved", C.c_int32 * 8)]


class ServerStats(C.Structure):
    """kf_server_stats_t (kf.h)."""
    _fields_ = [("frames", C.c_uint64), ("steps", C.c_uint64), ("busy_s", C.c_double),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("max_ms", C.c_double),
                ("bytes_in_use", C.c_uint64), ("active_sessions", C.c_int32), ("reserved", C.c_int32 * 7)]


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libkf.so and bind every entry point; raise if it or a symbol is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libkf.so not built: {path} (run python -m oglfusionkinectv2_b200.build)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)  # AttributeError if not exported
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def status_string(status: int) -> str:
    try:
        return load().kf_status_string(status).decode()
    except Exception:  # library absent: still describe the code
        return str(status)


def check(status: int, what: str) -> None:
    if status != KF_OK:
        raise KfError(status, what)
