"""ctypes binding of libkfb200.so (include/kf_api.h).

The library is loaded from ../lib next to this package.  There is no fallback: if the
shared library is missing the import fails with the build command to run.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(os.path.dirname(_HERE), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libkfb200.so")

KF_MAX_LEVELS = 3
KF_WEIGHT_SCALE = 1024.0

KF_OK = 0
KF_ERR_ARG = 1
KF_ERR_SHAPE = 2
KF_ERR_CUDA = 3
KF_ERR_NONFINITE = 4
KF_ERR_OOM_BUDGET = 5
KF_ERR_TIMEOUT = 6
KF_ERR_STATE = 7
KF_ERR_CAPACITY = 8
KF_ERR_TOO_LARGE = 9
KF_LLS_NOALLOC_MAX_ROWS = 1048576   # row limit of kf_solve_linear_least_squares_noalloc
KF_RENDER_NORMALS = 0
KF_RENDER_SHADING = 1
KF_DEBUG_RAY_TRACE = 1
KF_DEBUG_NO_GRAPH = 2
KF_DEBUG_COUNTERS = 4
KF_RAY_COUNTS = 8
RAY_COUNT_NAMES = ("rays", "eval_large", "eval_small", "skips", "skipped", "gradient", "queued", "long_rounds")
KF_MAX_FRAMES_IN_FLIGHT = 4

KF_TSDF_F32F32 = 0
KF_TSDF_F16U16 = 1


class KfConfig(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int),
        ("fx", ctypes.c_float), ("fy", ctypes.c_float), ("cx", ctypes.c_float), ("cy", ctypes.c_float),
        ("depth_scale", ctypes.c_float),
        ("unmirror", ctypes.c_int),
        ("levels", ctypes.c_int),
        ("iters", ctypes.c_int * KF_MAX_LEVELS),
        ("dist_thresh", ctypes.c_float), ("angle_thresh", ctypes.c_float),
        ("stop_angle", ctypes.c_float), ("stop_dist", ctypes.c_float),
        ("bilateral_sigma_s", ctypes.c_float), ("bilateral_sigma_r", ctypes.c_float),
        ("bilateral_radius", ctypes.c_int),
        ("volume_n", ctypes.c_int), ("volume_width", ctypes.c_float), ("mu", ctypes.c_float),
        ("max_weight", ctypes.c_float),
        ("tsdf_format", ctypes.c_int),
        ("min_depth", ctypes.c_float), ("max_depth", ctypes.c_float),
        ("step_large", ctypes.c_float), ("step_small", ctypes.c_float),
        ("compat_trunc8", ctypes.c_int), ("keep_on_miss", ctypes.c_int), ("export_icp_mask", ctypes.c_int),
        ("initial_pose", ctypes.c_float * 16),
        ("vis_volume_n", ctypes.c_int), ("vis_volume_width", ctypes.c_float), ("vis_mu", ctypes.c_float),
    ]


class KfVolume(ctypes.Structure):
    _fields_ = [
        ("f", ctypes.c_void_p), ("w", ctypes.c_void_p), ("n", ctypes.c_int),
        ("width", ctypes.c_float), ("mu", ctypes.c_float), ("format", ctypes.c_int),
        ("max_weight", ctypes.c_float),
    ]


class KfFrameStats(ctypes.Structure):
    _fields_ = [("frame", ctypes.c_int), ("status", ctypes.c_int), ("icp_iters", ctypes.c_int * KF_MAX_LEVELS)]


class KfServerStats(ctypes.Structure):
    _fields_ = [
        ("frames_done", ctypes.c_longlong), ("sessions_admitted", ctypes.c_longlong),
        ("sessions_refused", ctypes.c_longlong), ("steps", ctypes.c_longlong),
        ("active_sessions", ctypes.c_int), ("max_active_sessions", ctypes.c_int),
        ("hbm_in_use", ctypes.c_size_t), ("hbm_budget", ctypes.c_size_t),
        ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
    ]


_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_FP = ctypes.POINTER(ctypes.c_float)
_IP = ctypes.POINTER(ctypes.c_int)
_CFG = ctypes.POINTER(KfConfig)
_VOL = ctypes.POINTER(KfVolume)

# name -> (restype, argtypes); every function the header declares
SIGNATURES = {
    "kf_api_version": (_I, []),
    "kf_status_string": (ctypes.c_char_p, [_I]),
    "kf_config_default": (None, [_CFG]),
    "kf_session_footprint": (_I, [_CFG, ctypes.POINTER(ctypes.c_size_t)]),
    "kf_session_create": (_I, [_CFG, ctypes.POINTER(_P)]),
    "kf_session_destroy": (_I, [_P]),
    "kf_session_reset": (_I, [_P]),
    "kf_process_frame": (_I, [_P, _P, _I, _P, _FP]),
    "kf_process_frame_async": (_I, [_P, _P, _P]),
    "kf_process_frame_submit": (_I, [_P, _P, _I, _P]),
    "kf_process_frame_wait": (_I, [_P, _FP, ctypes.POINTER(KfFrameStats)]),
    "kf_get_pose": (_I, [_P, _FP]),
    "kf_set_pose": (_I, [_P, _FP]),
    "kf_get_frame_stats": (_I, [_P, ctypes.POINTER(KfFrameStats)]),
    "kf_get_depth": (_I, [_P, _I, _P, _I]),
    "kf_get_vertex": (_I, [_P, _I, _P, _I]),
    "kf_get_raycast": (_I, [_P, _I, _P, _P, _I]),
    "kf_get_icp_mask": (_I, [_P, _I, _P, _I]),
    "kf_get_tsdf": (_I, [_P, _P, ctypes.c_size_t, _I, _I]),
    "kf_set_tsdf": (_I, [_P, _P, ctypes.c_size_t, _I, _I]),
    "kf_get_volume": (_I, [_P, _VOL]),
    "kf_get_vis_tsdf": (_I, [_P, _P, ctypes.c_size_t, _I, _I]),
    "kf_get_vis_volume": (_I, [_P, _VOL]),
    "kf_convert_to_depth_meters": (_I, [_P, _I, _I, _P, _I, _I, _F, _I, _P, _FP]),
    "kf_apply_bilateral_filter": (_I, [_P, _I, _I, _P, _I, _I, _F, _F, _I, _P, _FP]),
    "kf_down_sample": (_I, [_P, _I, _I, _P, _I, _I, _F, _P, _FP]),
    "kf_create_vertex_map": (_I, [_P, _I, _I, _P, _I, _I, _FP, _P, _FP]),
    "kf_create_normal_map": (_I, [_P, _I, _I, _P, _I, _I, _P, _FP]),
    "kf_initialize_grid": (_I, [_VOL, _P, _FP]),
    "kf_fuse": (_I, [_P, _I, _I, _FP, _VOL, _FP, _F, _F, _P, _FP]),
    "kf_raycast": (_I, [_VOL, _FP, _FP, _P, _I, _I, _P, _I, _I, _F, _F, _F, _F, _P, _FP]),
    "kf_construct_icp_residuals": (_I, [_P, _P, _P, _I, _I, _FP, _FP, _FP, _FP, _FP, _F, _F, _P, _P, _P, _FP]),
    "kf_solve_linear_least_squares": (_I, [_P, _P, _I, _FP, _P]),
    "kf_solve_linear_least_squares_noalloc": (_I, [_P, _P, _I, _FP, _P]),
    "kf_compute_pose": (_I, [ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P), _I, _I, _I, _CFG, _FP, _FP,
                             _IP, _P]),
    "kf_pose_error": (_I, [_FP, _FP, _FP]),
    "kf_batch_create": (_I, [_CFG, _I, ctypes.POINTER(_P)]),
    "kf_batch_destroy": (_I, [_P]),
    "kf_batch_step": (_I, [_P, ctypes.POINTER(_P), _I, _P, _FP]),
    "kf_batch_step_async": (_I, [_P, _IP, _P]),
    "kf_batch_input_buffer": (_I, [_P, _I, ctypes.POINTER(_P)]),
    "kf_batch_session": (_I, [_P, _I, ctypes.POINTER(_P)]),
    "kf_batch_autotune_start": (_I, [_P, ctypes.c_char_p]),
    "kf_batch_autotune_status": (_I, [_P, _IP, ctypes.c_char_p, ctypes.c_size_t]),
    "kf_server_create": (_I, [_I, ctypes.c_size_t, ctypes.POINTER(_P)]),
    "kf_server_destroy": (_I, [_P]),
    "kf_server_open": (_I, [_P, _CFG, _IP]),
    "kf_server_close": (_I, [_P, _I]),
    "kf_server_submit": (_I, [_P, _I, _P, ctypes.c_double]),
    "kf_server_step": (_I, [_P, _IP]),
    "kf_server_result": (_I, [_P, _I, _FP, ctypes.POINTER(KfFrameStats)]),
    "kf_server_get_session": (_I, [_P, _I, ctypes.POINTER(_P)]),
    "kf_server_stats_get": (_I, [_P, ctypes.POINTER(KfServerStats)]),
    "kf_server_stats_reset": (_I, [_P]),
    "kf_server_reserve": (_I, [_P, _CFG, _I]),
    "kf_save_tsdf_file": (_I, [_P, ctypes.c_char_p]),
    "kf_load_tsdf_file": (_I, [_P, ctypes.c_char_p]),
    "kf_save_vis_tsdf_file": (_I, [_P, ctypes.c_char_p]),
    "kf_load_vis_tsdf_file": (_I, [_P, ctypes.c_char_p]),
    "kf_session_checkpoint_save": (_I, [_P, ctypes.c_char_p]),
    "kf_session_checkpoint_load": (_I, [_P, ctypes.c_char_p]),
    "kf_normal_map_to_rgba": (_I, [_P, _I, _I, _FP, _P, _P, _FP]),
    "kf_shading_to_rgba": (_I, [_P, _I, _I, _FP, _FP, _P, _P, _FP]),
    "kf_float_channel_to_rgba": (_I, [_P, _I, _I, _F, _P, _P, _FP]),
    "kf_render": (_I, [_P, _I, _FP, _P, _I, _P]),
    "kf_tum_open": (_I, [ctypes.c_char_p, ctypes.POINTER(_P)]),
    "kf_tum_close": (_I, [_P]),
    "kf_tum_count": (_I, [_P, _IP]),
    "kf_tum_frame": (_I, [_P, _I, _P, _I, _I, _FP]),
    "kf_tum_initial_pose_inverse": (_I, [_P, _FP]),
    "kf_png16_read": (_I, [ctypes.c_char_p, _P, _I, _I]),
    "kf_now_ms": (ctypes.c_double, []),
    "kf_session_set_profiling": (_I, [_P, _I]),
    "kf_session_stage_times": (_I, [_P, _FP]),
    "kf_session_set_debug": (_I, [_P, _I]),
    "kf_batch_set_debug": (_I, [_P, _I]),
    "kf_session_debug_counts": (_I, [_P, _P, _I]),
    "kf_batch_debug_counts": (_I, [_P, _P, _I]),
    "kf_get_ray_trace": (_I, [_P, _I, _P, _I]),
    "kf_batch_set_profiling": (_I, [_P, _I]),
    "kf_batch_stage_times": (_I, [_P, _FP]),
    "kf_selftest_bounded_wait": (_I, [_I, _IP]),
    "kf_measure_read_bandwidth": (_I, [ctypes.c_size_t, _I, ctypes.POINTER(ctypes.c_double)]),
}


def load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "libkfb200.so is not built (%s); run `python kinectfusion-cuda_b200/build.py` "
            "(or __graft_entry__.build())" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = load()


class KfError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = lib.kf_status_string(status).decode()
        super().__init__("%s: %s (status %d)" % (what, msg, status) if what else "%s (status %d)" % (msg, status))


def check(status, what=""):
    if status != KF_OK:
        raise KfError(status, what)
    return status
