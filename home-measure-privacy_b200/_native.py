"""ctypes binding of libgsb200.so, the C ABI declared in include/gsb200.h.

Loading fails loudly when the library has not been built: there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgsb200.so")

GS_OK = 0
GS_ERR_INVALID_ARG = -1
GS_ERR_CUDA = -2
GS_ERR_CAPACITY = -3
GS_ERR_NO_DEVICE = -4
GS_ERR_STATE = -5
GS_ERR_NONFINITE = -6
GS_NUM_STAGES = 10

c_float, c_int32, c_int64 = ctypes.c_float, ctypes.c_int32, ctypes.c_int64


class GsCamera(ctypes.Structure):
    _fields_ = [("view", c_float * 12), ("fx", c_float), ("fy", c_float), ("cx", c_float), ("cy", c_float),
                ("width", c_int32), ("height", c_int32)]


class GsConfig(ctypes.Structure):
    _fields_ = [("near_plane", c_float), ("cov_dilation", c_float), ("alpha_max", c_float),
                ("alpha_min", c_float), ("t_min", c_float), ("sh_degree", c_int32), ("rect_mode", c_int32),
                ("batched", c_int32), ("use_graph", c_int32), ("device", c_int32), ("autotune", c_int32),
                ("raster_batch", c_int32), ("lpt_order", c_int32), ("instance_capacity", c_int32),
                ("raster_ppt", c_int32), ("tile_cull", c_int32), ("tile_size", c_int32),
                ("raster_work_tile", c_int32)]


class GsAdamConfig(ctypes.Structure):
    _fields_ = [("lr_color", c_float), ("lr_opacity", c_float), ("lr_mean", c_float), ("lr_scale", c_float),
                ("lr_rotation", c_float), ("lr_sh", c_float), ("beta1", c_float), ("beta2", c_float),
                ("eps", c_float)]


class GsLossConfig(ctypes.Structure):
    _fields_ = [("ssim_lambda", c_float), ("window", c_int32)]


class GsStats(ctypes.Structure):
    _fields_ = [("instances", c_int64), ("instance_capacity", c_int64), ("visible_pairs", c_int64),
                ("tiles", c_int64), ("pixels", c_int64), ("kernel_launches_per_step", c_int64),
                ("raster_batch", c_int32), ("raster_threads", c_int32), ("overflow", c_int32),
                ("raster_variant", c_int32), ("tile_size", c_int32)]


class GsError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


F32P = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
U8P = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
VP = ctypes.c_void_p
CTX = ctypes.c_void_p

# name -> (restype, argtypes)
GRAD_TAIL_FLOATS = 64  # GS_GRAD_TAIL_FLOATS


class GsDensifyConfig(ctypes.Structure):
    _fields_ = [("grad_threshold", ctypes.c_double), ("size_threshold", ctypes.c_double),
                ("min_opacity", ctypes.c_double), ("max_size", ctypes.c_double), ("max_count", c_int32),
                ("reserved", c_int32), ("seed", ctypes.c_uint64)]

SIGNATURES = {
    "gs_config_default": (None, [ctypes.POINTER(GsConfig)]),
    "gs_adam_default": (None, [ctypes.POINTER(GsAdamConfig)]),
    "gs_create": (ctypes.c_int, [ctypes.POINTER(GsConfig), ctypes.POINTER(CTX)]),
    "gs_destroy": (ctypes.c_int, [CTX]),
    "gs_last_error": (ctypes.c_char_p, []),
    "gs_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "gs_param_stride": (ctypes.c_int, [ctypes.c_int]),
    "gs_set_gaussians": (ctypes.c_int, [CTX, c_int32, VP]),
    "gs_set_gaussians_packed": (ctypes.c_int, [CTX, c_int32, VP]),
    "gs_get_gaussians": (ctypes.c_int, [CTX, VP]),
    "gs_get_gaussians_packed": (ctypes.c_int, [CTX, VP]),
    "gs_num_gaussians": (c_int32, [CTX]),
    "gs_set_views": (ctypes.c_int, [CTX, c_int32, ctypes.POINTER(GsCamera)]),
    "gs_set_target_u8": (ctypes.c_int, [CTX, c_int32, VP]),
    "gs_set_target_f32": (ctypes.c_int, [CTX, c_int32, VP]),
    "gs_render": (ctypes.c_int, [CTX, ctypes.POINTER(GsCamera), VP, VP]),
    "gs_forward": (ctypes.c_int, [CTX, c_int32, c_int32, VP]),
    "gs_backward": (ctypes.c_int, [CTX, VP]),
    "gs_loss": (ctypes.c_int, [CTX, ctypes.POINTER(GsLossConfig), ctypes.POINTER(c_float)]),
    "gs_get_param_grads": (ctypes.c_int, [CTX, VP]),
    "gs_get_screen_grads": (ctypes.c_int, [CTX, c_int32, VP]),
    "gs_gradients": (ctypes.c_int, [CTX, ctypes.POINTER(GsCamera), VP, c_float, VP, VP, VP]),
    "gs_loss_gradient": (ctypes.c_int, [CTX, VP, VP, c_int32, c_int32, c_float, c_int32, VP,
                                        ctypes.POINTER(c_float)]),
    "gs_train_step": (ctypes.c_int, [CTX, ctypes.POINTER(GsAdamConfig), ctypes.POINTER(GsLossConfig), c_int32,
                                     c_int32, ctypes.POINTER(c_float)]),
    "gs_train_step_host": (ctypes.c_int, [CTX, ctypes.POINTER(GsAdamConfig), ctypes.POINTER(GsLossConfig),
                                          c_int32, c_int32, VP, ctypes.POINTER(c_float)]),
    "gs_train": (ctypes.c_int, [CTX, c_int32, ctypes.POINTER(GsAdamConfig), VP]),
    "gs_get_step": (ctypes.c_int, [CTX, ctypes.POINTER(c_int32)]),
    "gs_debug_lookback_wait": (ctypes.c_int, [CTX, c_int32]),
    "gs_train_step_host_async": (ctypes.c_int, [CTX, ctypes.POINTER(GsAdamConfig), ctypes.POINTER(GsLossConfig),
                                                c_int32, c_int32, VP, VP]),
    "gs_step_gradients": (ctypes.c_int, [CTX, ctypes.POINTER(GsLossConfig), c_int32, c_int32,
                                         ctypes.POINTER(ctypes.POINTER(c_float)), ctypes.POINTER(ctypes.c_int64)]),
    "gs_step_apply": (ctypes.c_int, [CTX, ctypes.POINTER(GsAdamConfig), ctypes.POINTER(c_float),
                                     ctypes.POINTER(c_int32)]),
    "gs_get_stream": (ctypes.c_int, [CTX, ctypes.POINTER(VP)]),
    "gs_dp_unique_id": (ctypes.c_int, [VP, c_int32]),
    "gs_dp_init": (ctypes.c_int, [CTX, VP, c_int32, c_int32, c_int32]),
    "gs_dp_allreduce": (ctypes.c_int, [CTX]),
    "gs_dp_finalize": (ctypes.c_int, [CTX]),
    "gs_get_blend_count": (ctypes.c_int, [CTX, ctypes.POINTER(ctypes.c_uint64)]),
    "gs_neighbour_sizes": (ctypes.c_int, [CTX, VP, c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double, VP]),
    "gs_init_from_points": (ctypes.c_int, [CTX, VP, VP, c_int32, c_float]),
    "gs_sharpness": (ctypes.c_int, [CTX, VP, c_int32, c_int32, c_int32, c_int32, VP]),
    "gs_choose_sharp": (ctypes.c_int, [VP, c_int32, c_int32, VP, ctypes.POINTER(c_int32)]),
    "gs_load_ply": (ctypes.c_int, [CTX, VP, ctypes.c_int64, ctypes.POINTER(c_int32)]),
    "gs_save_ply": (ctypes.c_int, [CTX, c_int32, VP, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    "gs_save_splat": (ctypes.c_int, [CTX, VP, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    "gs_set_densify_stats": (ctypes.c_int, [CTX, c_int32]),
    "gs_reset_densify_stats": (ctypes.c_int, [CTX]),
    "gs_get_densify_stats": (ctypes.c_int, [CTX, VP, VP]),
    "gs_densify_config_default": (None, [ctypes.POINTER(GsDensifyConfig)]),
    "gs_densify": (ctypes.c_int, [CTX, ctypes.POINTER(GsDensifyConfig), ctypes.POINTER(c_int32)]),
    "gs_reset_opacity": (ctypes.c_int, [CTX, ctypes.c_double]),
    "gs_scene_extent": (ctypes.c_int, [ctypes.POINTER(GsCamera), c_int32, ctypes.POINTER(c_float)]),
    "gs_host_alloc": (ctypes.c_int, [ctypes.c_size_t, ctypes.POINTER(VP)]),
    "gs_host_free": (ctypes.c_int, [VP]),
    "gs_synchronize": (ctypes.c_int, [CTX]),
    "gs_event_record": (ctypes.c_int, [CTX, c_int32]),
    "gs_event_elapsed": (ctypes.c_int, [CTX, c_int32, c_int32, ctypes.POINTER(c_float)]),
    "gs_stage_name": (ctypes.c_char_p, [c_int32]),
    "gs_stage_times": (ctypes.c_int, [CTX, VP, VP, ctypes.POINTER(c_int32)]),
    "gs_stage_times_reset": (ctypes.c_int, [CTX]),
    "gs_set_stage_timing": (ctypes.c_int, [CTX, c_int32]),
    "gs_get_stats": (ctypes.c_int, [CTX, ctypes.POINTER(GsStats)]),
    "gs_get_tile_lists": (ctypes.c_int, [CTX, c_int32, VP, VP, VP, c_int64, ctypes.POINTER(c_int64)]),
    "gs_get_splats": (ctypes.c_int, [CTX, c_int32, VP]),
    "gs_autotune": (ctypes.c_int, [CTX, ctypes.c_char_p]),
    "gs_loss_gradient_noalloc": (ctypes.c_int, [VP, VP, c_int32, c_int32, c_int32, c_float, c_int32, VP, VP, VP]),
}

_lib = None


def load(path=LIB_PATH):
    """Load libgsb200.so and declare every signature.  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python {os.path.join(HERE, 'build.py')}` "
                           "(the CUDA library is required; there is no CPU fallback)")
    L = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status):
    if status != GS_OK:
        L = load()
        raise GsError(status, L.gs_last_error().decode())
    return status


def ptr(a):
    """Data pointer of a contiguous numpy array (None for None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data
