"""ctypes binding of libdroplet_b200.so (declarations: include/droplet_b200.h).

The shared library is the product: there is no CPU fallback.  If it is
missing or cannot be loaded this module raises, so a GPU box never silently
runs something else.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdroplet_b200.so")

DL_OK, DL_E_INVALID_ARG, DL_E_OOM, DL_E_CUDA, DL_E_TIMEOUT, DL_E_CAPACITY, DL_E_NO_DEVICE = range(7)
DL_PINHOLE, DL_EQUIRECT = 0, 1
DL_PREC_F32, DL_PREC_F16, DL_PREC_BF16 = 0, 1, 2
DL_BATCH_OUT_DEVICE = 1
DL_BATCH_PLAIN = 2
DL_BATCH_F16_RECORDS = 4
DL_BATCH_NO_GRAPH = 8
DL_BATCH_STATIC = 16
DL_BATCH_FAST_EXP = 32
DL_BATCH_COUNT_EVALS = 64
DL_BATCH_LOG_TILES = 128
DL_BATCH_F64_DEGENERATE = 256
DL_BATCH_SH16 = 512
DL_BATCH_CULL_OFFSCREEN = 1024
DL_PLY_PINNED = 1
DL_VOX_FAST_EXP = 1
DL_VOX_PROFILE = 2
DL_MLP_IN, DL_MLP_HIDDEN = 12, 64
DL_MLP_PARAMS = 12 * 64 + 64 + 64 * 64 + 64 + 64 + 1

# Every function the header declares (checked by the CPU test suite).
EXPORTS = [
    "dl_last_error", "dl_device_open", "dl_device_close", "dl_renderer_create", "dl_renderer_destroy",
    "dl_renderer_set_stream", "dl_render", "dl_scene_upload", "dl_scene_free", "dl_render_batch",
    "dl_voxelize", "dl_vox_result_info", "dl_vox_result_copy", "dl_vox_result_free",
    "dl_renderer_debug_get", "dl_renderer_set_profiling", "dl_renderer_stage_times",
    "dl_renderer_launch_count", "dl_renderer_set_debug", "dl_render_many",
    "dl_render_static", "dl_mlp_create", "dl_mlp_destroy", "dl_mlp_get_params", "dl_mlp_set_params",
    "dl_mlp_predict", "dl_mlp_grad", "dl_mlp_train", "dl_renderer_set_scheduler", "dl_renderer_tile_log",
    "dl_sorter_create", "dl_sorter_destroy", "dl_sorter_set_stream", "dl_sorter_set_digit_bits", "dl_sorter_sort",
    "dl_renderer_set_tuning", "dl_renderer_get_tuning", "dl_renderer_autotune",
    "dl_device_set_voxel_scheduler", "dl_vox_result_block_log", "dl_test_set_wait_limit",
    "dl_test_withhold_status", "dl_test_fail_allocation", "dl_ply_load", "dl_ply_splats", "dl_ply_free",
    "dl_vox_result_stage_times", "dl_vox_query", "dl_vox_carve",
]


class DlSplats(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint64),
                ("positions", ctypes.c_void_p), ("rotations", ctypes.c_void_p),
                ("log_scales", ctypes.c_void_p), ("opacity_logits", ctypes.c_void_p),
                ("colors_dc", ctypes.c_void_p), ("colors_sh", ctypes.c_void_p),
                ("sh_bands", ctypes.c_int32)]


class DlCamera(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("view", ctypes.c_float * 16),
                ("fov_y", ctypes.c_double), ("near_plane", ctypes.c_double), ("far_plane", ctypes.c_double),
                ("projection", ctypes.c_int32)]


class DlRendererOpts(ctypes.Structure):
    _fields_ = [("chunk_cap", ctypes.c_uint32), ("max_coverage_per_splat", ctypes.c_uint32)]


class DlTuning(ctypes.Structure):
    _fields_ = [("pair_sort_bits", ctypes.c_int32), ("raster_shape", ctypes.c_int32),
                ("raster_ctas_per_sm", ctypes.c_int32), ("bin_tile", ctypes.c_int32)]


class DlVoxOpts(ctypes.Structure):
    _fields_ = [("voxel_resolution", ctypes.c_double), ("opacity_cutoff", ctypes.c_double),
                ("use_defaults", ctypes.c_int32), ("has_bounds", ctypes.c_int32),
                ("bounds_min", ctypes.c_double * 3), ("bounds_max", ctypes.c_double * 3),
                ("shard_index", ctypes.c_int32), ("shard_count", ctypes.c_int32), ("log_blocks", ctypes.c_int32),
                ("flags", ctypes.c_uint32)]


_lib = None
vp = ctypes.c_void_p
P = ctypes.POINTER


def load():
    """Load the library (building it first if the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH) or os.environ.get("DL_REBUILD"):
        from . import build as _build
        _build.build()
    L = ctypes.CDLL(LIB_PATH)
    i = ctypes.c_int
    L.dl_last_error.restype = ctypes.c_char_p
    L.dl_last_error.argtypes = []
    sigs = {
        "dl_device_open": [i, P(vp)],
        "dl_device_close": [vp],
        "dl_renderer_create": [vp, P(DlRendererOpts), P(vp)],
        "dl_renderer_destroy": [vp],
        "dl_renderer_set_stream": [vp, vp],
        "dl_render": [vp, P(DlSplats), P(DlCamera), P(ctypes.c_float), vp, ctypes.c_size_t],
        "dl_scene_upload": [vp, P(DlSplats), i, P(vp)],
        "dl_scene_free": [vp],
        "dl_render_batch": [vp, vp, P(DlCamera), i, P(ctypes.c_float), P(vp), ctypes.c_uint32],
        "dl_render_many": [vp, P(DlSplats), P(DlCamera), i, P(ctypes.c_float), P(vp), ctypes.c_uint32],
        "dl_render_static": [P(DlSplats), P(DlCamera), P(ctypes.c_float), ctypes.c_uint32, vp, ctypes.c_size_t],
        "dl_mlp_create": [vp, ctypes.c_uint64, P(vp)],
        "dl_mlp_destroy": [vp],
        "dl_mlp_get_params": [vp, vp, ctypes.c_size_t],
        "dl_mlp_set_params": [vp, vp, ctypes.c_size_t],
        "dl_mlp_predict": [vp, vp, ctypes.c_uint64, vp],
        "dl_mlp_grad": [vp, vp, vp, ctypes.c_uint64, vp, P(ctypes.c_float)],
        "dl_mlp_train": [vp, vp, vp, ctypes.c_uint64, i, i, ctypes.c_float, ctypes.c_uint64, P(ctypes.c_float)],
        "dl_renderer_set_scheduler": [vp, vp],
        "dl_renderer_tile_log": [vp, vp, vp, ctypes.c_uint64, P(ctypes.c_uint64)],
        "dl_voxelize": [vp, P(DlSplats), P(DlVoxOpts), P(vp)],
        "dl_vox_result_info": [vp, P(ctypes.c_double), P(ctypes.c_double), P(ctypes.c_double), P(ctypes.c_uint64)],
        "dl_vox_result_copy": [vp, vp, vp, vp],
        "dl_vox_result_free": [vp],
        "dl_renderer_debug_get": [vp, ctypes.c_char_p, vp, ctypes.c_size_t, P(ctypes.c_size_t)],
        "dl_renderer_set_profiling": [vp, i],
        "dl_renderer_stage_times": [vp, P(ctypes.c_double), i],
        "dl_renderer_launch_count": [vp, P(ctypes.c_uint64)],
        "dl_renderer_set_debug": [vp, i],
        "dl_sorter_create": [vp, P(vp)],
        "dl_sorter_destroy": [vp],
        "dl_sorter_set_stream": [vp, vp],
        "dl_sorter_set_digit_bits": [vp, i],
        "dl_sorter_sort": [vp, vp, vp, ctypes.c_uint64, ctypes.c_uint32, P(vp), P(vp)],
        "dl_renderer_set_tuning": [vp, P(DlTuning)],
        "dl_device_set_voxel_scheduler": [vp, vp],
        "dl_vox_result_block_log": [vp, vp, vp, ctypes.c_uint64, P(ctypes.c_uint64)],
        "dl_renderer_get_tuning": [vp, P(DlTuning)],
        "dl_test_set_wait_limit": [ctypes.c_uint32],
        "dl_test_withhold_status": [i, ctypes.c_uint32],
        "dl_test_fail_allocation": [i],
        "dl_ply_load": [vp, ctypes.c_size_t, i, ctypes.c_uint32, P(vp)],
        "dl_ply_splats": [vp, P(DlSplats)],
        "dl_ply_free": [vp],
        "dl_vox_result_stage_times": [vp, P(ctypes.c_double), i],
        "dl_vox_query": [vp, vp, vp, vp, ctypes.c_uint64, P(ctypes.c_double), ctypes.c_double, P(ctypes.c_double),
                         vp, ctypes.c_uint64, vp],
        "dl_vox_carve": [vp, vp, vp, vp, ctypes.c_uint64, vp, vp, vp, ctypes.c_uint64, vp, vp, vp, P(ctypes.c_uint64)],
        "dl_renderer_autotune": [vp, vp, P(DlCamera), i, P(ctypes.c_float), ctypes.c_uint32, i, P(DlTuning),
                                 P(ctypes.c_double)],
    }
    for name, args in sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    _lib = L
    return L


class DropletError(RuntimeError):
    """Raised for a non-zero status; carries the code and dl_last_error()."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def check(status: int):
    if status != DL_OK:
        raise DropletError(status, load().dl_last_error().decode(errors="replace"))
