"""ctypes binding of libimogen_b200.so (the C ABI declared in include/imogen_b200.h).

The library is built in-tree (imogen_b200/build.py).  There is no fallback: if the shared library
is missing or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libimogen_b200.so")

# status codes (include/imogen_b200.h)
IMG_OK = 0
STATUS = {
    -1: "IMG_ERR_ARG", -2: "IMG_ERR_CUDA", -3: "IMG_ERR_NOMEM", -4: "IMG_ERR_UNSUPPORTED",
    -5: "IMG_ERR_CFL", -6: "IMG_ERR_NONFINITE", -7: "IMG_ERR_STATE",
}

# exported symbols, in header order
SYMBOLS = (
    "img_config_default", "img_create", "img_destroy", "img_set_state", "img_upload", "img_download",
    "img_upload_many", "img_download_many",
    "img_time_update", "img_flux", "img_fluid_sweep", "img_magnet_sweep", "img_step", "img_run",
    "img_get_time", "img_set_time", "img_progress", "img_checkpoint_bytes", "img_checkpoint_save",
    "img_checkpoint_load", "img_totals", "img_totals_static", "img_sync", "img_last_error", "img_bytes_required",
    "img_get_stream", "img_autotune", "img_get_tiling", "img_set_tiling", "img_launch_count", "img_sweep_order",
    "img_source", "img_radiation_strength", "img_treadmill", "img_treadmill_history",
    "img_slice_write", "img_slice_read", "img_slice_last_error", "img_save_slice", "img_load_slice",
    "img_server_create", "img_server_destroy", "img_batch_submit", "img_batch_poll", "img_batch_cancel",
    "img_batch_result", "img_server_stats", "img_monotonic_seconds",
    "img_batch_create", "img_batch_destroy", "img_batch_add", "img_batch_remove", "img_batch_size", "img_batch_step",
    "img_batch_run", "img_batch_status", "img_batch_get_stream", "img_batch_launch_count", "img_batch_last_error",
)


class ImgConfig(ctypes.Structure):
    _fields_ = [
        ("grid", ctypes.c_int * 3),
        ("dgrid", ctypes.c_double * 3),
        ("gamma", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("minmass", ctypes.c_double),
        ("bc_infinity", ctypes.c_int),
        ("bc_modes", ((ctypes.c_int * 3) * 2) * 4),
        ("limiter", ctypes.c_int * 3),
        ("fluid_active", ctypes.c_int),
        ("magnet_active", ctypes.c_int),
        ("time_max", ctypes.c_double),
        ("iter_max", ctypes.c_int),
        ("update_mode", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("nonfinite_check", ctypes.c_int),
        ("viscosity_type", ctypes.c_int),
        ("visc_linear", ctypes.c_double),
        ("visc_quadratic", ctypes.c_double),
        ("radiation_type", ctypes.c_int),
        ("rad_exponent", ctypes.c_double),
        ("rad_initial_maximum", ctypes.c_double),
        ("treadmill", ctypes.c_int),
        ("fade_active", ctypes.c_int),
        ("fade_location", ctypes.c_int * 3),
        ("fade_size", ctypes.c_double),
    ]


class ImgSliceMeta(ctypes.Structure):
    _fields_ = [
        ("type", ctypes.c_int),
        ("index", ctypes.c_int * 3),
        ("suffix", ctypes.c_char_p),
        ("about", ctypes.c_char_p),
        ("version", ctypes.c_double),
        ("wall_max", ctypes.c_double),
        ("started", ctypes.c_char_p),
    ]


class ImgSliceState(ctypes.Structure):
    _fields_ = [
        ("grid", ctypes.c_int * 3),
        ("dgrid", ctypes.c_double * 3),
        ("gamma", ctypes.c_double),
        ("time", ctypes.c_double),
        ("iteration", ctypes.c_int),
        ("iter_max", ctypes.c_int),
        ("time_max", ctypes.c_double),
        ("dt_history", ctypes.POINTER(ctypes.c_double)),
        ("n_history", ctypes.c_int),
        ("magnet_active", ctypes.c_int),
        ("mass", ctypes.POINTER(ctypes.c_double)),
        ("mom", ctypes.POINTER(ctypes.c_double)),
        ("ener", ctypes.POINTER(ctypes.c_double)),
        ("mag", ctypes.POINTER(ctypes.c_double)),
        ("treadmill", ctypes.c_int),
        ("tread_history", ctypes.POINTER(ctypes.c_int)),
        ("n_tread", ctypes.c_int),
    ]


class ImgJobInfo(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int),
        ("time", ctypes.c_double),
        ("iterations", ctypes.c_int),
        ("submitted", ctypes.c_double),
        ("admitted", ctypes.c_double),
        ("completed", ctypes.c_double),
        ("error_code", ctypes.c_int),
        ("error", ctypes.c_char * 256),
    ]


class ImgServerInfo(ctypes.Structure):
    _fields_ = [
        ("budget", ctypes.c_size_t),
        ("used", ctypes.c_size_t),
        ("peak", ctypes.c_size_t),
        ("queued", ctypes.c_int),
        ("running", ctypes.c_int),
        ("finished", ctypes.c_int),
        ("rounds", ctypes.c_longlong),
    ]


class ImogenError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


_LIB = None


def lib():
    """Load libimogen_b200.so (building it first if it is absent and nvcc is available)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    from . import build
    build.build()   # no-op when libimogen_b200.so is newer than its sources
    L = ctypes.CDLL(LIB_PATH)
    vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    cfgp = ctypes.POINTER(ImgConfig)
    L.img_config_default.argtypes = [cfgp]
    L.img_config_default.restype = None
    L.img_create.argtypes = [ctypes.POINTER(vp), cfgp]
    L.img_destroy.argtypes = [vp]
    L.img_set_state.argtypes = [vp, dp, dp, dp, dp]
    L.img_upload.argtypes = [vp, ctypes.c_int, dp, ctypes.c_size_t]
    L.img_download.argtypes = [vp, ctypes.c_int, dp, ctypes.c_size_t]
    L.img_upload_many.argtypes = [vp, ctypes.c_int, ip, ctypes.POINTER(dp), ctypes.c_size_t]
    L.img_upload_many.restype = ctypes.c_int
    L.img_download_many.argtypes = [vp, ctypes.c_int, ip, ctypes.POINTER(dp), ctypes.c_size_t]
    L.img_download_many.restype = ctypes.c_int
    L.img_time_update.argtypes = [vp, ctypes.c_int, dp, ip]
    L.img_flux.argtypes = [vp, ctypes.c_int]
    L.img_fluid_sweep.argtypes = [vp, ctypes.c_int]
    L.img_magnet_sweep.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.img_step.argtypes = [vp]
    L.img_run.argtypes = [vp, ctypes.c_int, ip]
    L.img_get_time.argtypes = [vp, dp, dp, ip]
    L.img_set_time.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    L.img_totals.argtypes = [vp, dp]
    L.img_progress.argtypes = [vp, dp, ip, ip]
    L.img_checkpoint_bytes.argtypes = [vp]
    L.img_checkpoint_bytes.restype = ctypes.c_size_t
    L.img_checkpoint_save.argtypes = [vp, vp, ctypes.c_size_t]
    L.img_checkpoint_save.restype = ctypes.c_int
    L.img_checkpoint_load.argtypes = [vp, vp, ctypes.c_size_t]
    L.img_checkpoint_load.restype = ctypes.c_int
    L.img_progress.restype = ctypes.c_int
    L.img_totals_static.argtypes = [vp, dp]
    L.img_sync.argtypes = [vp]
    L.img_last_error.argtypes = [vp]
    L.img_last_error.restype = ctypes.c_char_p
    L.img_bytes_required.argtypes = [cfgp]
    L.img_bytes_required.restype = ctypes.c_size_t
    L.img_get_stream.argtypes = [vp, ctypes.POINTER(ctypes.c_void_p)]
    L.img_get_stream.restype = ctypes.c_int
    L.img_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64)]
    L.img_autotune.argtypes = [vp, ctypes.c_int]
    L.img_autotune.restype = ctypes.c_int
    L.img_get_tiling.argtypes = [vp, ctypes.c_int, ip]
    L.img_get_tiling.restype = ctypes.c_int
    L.img_set_tiling.argtypes = [vp, ctypes.c_int, ip]
    L.img_set_tiling.restype = ctypes.c_int
    L.img_launch_count.restype = ctypes.c_int
    L.img_sweep_order.argtypes = [ctypes.c_int, ctypes.c_int, ip]
    L.img_sweep_order.restype = ctypes.c_int
    L.img_source.argtypes = [vp]
    L.img_source.restype = ctypes.c_int
    L.img_radiation_strength.argtypes = [vp, dp]
    L.img_radiation_strength.restype = ctypes.c_int
    L.img_treadmill.argtypes = [vp]
    L.img_treadmill.restype = ctypes.c_int
    L.img_treadmill_history.argtypes = [vp, ip, ctypes.c_int, ip, ip]
    L.img_treadmill_history.restype = ctypes.c_int
    L.img_slice_write.argtypes = [ctypes.c_char_p, ctypes.POINTER(ImgSliceMeta), ctypes.POINTER(ImgSliceState)]
    L.img_slice_write.restype = ctypes.c_int
    L.img_slice_read.argtypes = [ctypes.c_char_p, ip, dp, dp, dp, dp, ip]
    L.img_slice_read.restype = ctypes.c_int
    L.img_slice_last_error.argtypes = []
    L.img_slice_last_error.restype = ctypes.c_char_p
    L.img_save_slice.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ImgSliceMeta)]
    L.img_save_slice.restype = ctypes.c_int
    L.img_load_slice.argtypes = [vp, ctypes.c_char_p]
    L.img_load_slice.restype = ctypes.c_int
    L.img_server_create.argtypes = [ctypes.POINTER(vp), ctypes.c_size_t, ctypes.c_int, ctypes.c_int]
    L.img_server_destroy.argtypes = [vp]
    L.img_batch_submit.argtypes = [vp, cfgp, dp, dp, dp, dp, ip]
    L.img_batch_poll.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ImgJobInfo)]
    L.img_batch_cancel.argtypes = [vp, ctypes.c_int]
    L.img_batch_result.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_size_t]
    L.img_server_stats.argtypes = [vp, ctypes.POINTER(ImgServerInfo)]
    for name in ("img_server_create", "img_server_destroy", "img_batch_submit", "img_batch_poll", "img_batch_cancel",
                 "img_batch_result", "img_server_stats"):
        getattr(L, name).restype = ctypes.c_int
    L.img_monotonic_seconds.argtypes = []
    L.img_monotonic_seconds.restype = ctypes.c_double
    L.img_batch_create.argtypes = [ctypes.POINTER(vp)]
    L.img_batch_destroy.argtypes = [vp]
    L.img_batch_add.argtypes = [vp, vp]
    L.img_batch_remove.argtypes = [vp, vp]
    L.img_batch_size.argtypes = [vp, ip]
    L.img_batch_step.argtypes = [vp]
    L.img_batch_run.argtypes = [vp, ctypes.c_int, ctypes.c_int, ip]
    L.img_batch_status.argtypes = [vp, ip, ctypes.c_int]
    L.img_batch_get_stream.argtypes = [vp, ctypes.POINTER(ctypes.c_void_p)]
    L.img_batch_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64)]
    L.img_batch_last_error.argtypes = [vp]
    L.img_batch_last_error.restype = ctypes.c_char_p
    for name in ("img_batch_create", "img_batch_destroy", "img_batch_add", "img_batch_remove", "img_batch_size",
                 "img_batch_step", "img_batch_run", "img_batch_status", "img_batch_get_stream",
                 "img_batch_launch_count"):
        getattr(L, name).restype = ctypes.c_int
    for name in ("img_create", "img_destroy", "img_set_state", "img_upload", "img_download",
                 "img_time_update", "img_flux", "img_fluid_sweep", "img_magnet_sweep", "img_step",
                 "img_run", "img_get_time", "img_set_time", "img_totals", "img_totals_static", "img_sync"):
        getattr(L, name).restype = ctypes.c_int
    _LIB = L
    return L


def check(rc, ctx=None):
    if rc != IMG_OK:
        msg = lib().img_last_error(ctx)
        raise ImogenError(rc, msg.decode() if msg else "")
    return rc
