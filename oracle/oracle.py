"""ORACLE — test infrastructure only.

ctypes front end for oracle/_build/liboracle.so, the C++ restatement of the
reference's render and voxelize paths (oracle_render.cpp, oracle_voxel.cpp).
Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it,
always as the checker; the product package never imports it.

Parity unpinned: the reference (TypeScript over WebGPU) cannot run here and publishes no
numeric vectors; the oracle is checked by closed-form known answers
(tests/golden/kat.json) and the reference's qualitative checks.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


class OrcSplats(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint64),
                ("positions", ctypes.c_void_p), ("rotations", ctypes.c_void_p),
                ("log_scales", ctypes.c_void_p), ("opacity_logits", ctypes.c_void_p),
                ("colors_dc", ctypes.c_void_p), ("colors_sh", ctypes.c_void_p),
                ("sh_bands", ctypes.c_int32)]


class OrcCamera(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("view", ctypes.c_float * 16),
                ("fov_y", ctypes.c_double), ("near_plane", ctypes.c_double), ("far_plane", ctypes.c_double),
                ("projection", ctypes.c_int32)]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_render_run.restype = ctypes.c_void_p
        L.orc_render_run.argtypes = [ctypes.POINTER(OrcSplats), ctypes.POINTER(OrcCamera), ctypes.c_uint32,
                                     ctypes.c_uint32, ctypes.POINTER(ctypes.c_float), ctypes.c_int]
        L.orc_render_get.restype = ctypes.c_int64
        L.orc_render_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int64]
        L.orc_render_free.argtypes = [ctypes.c_void_p]
        L.orc_voxelize_run.restype = ctypes.c_void_p
        L.orc_voxelize_run.argtypes = [ctypes.POINTER(OrcSplats), ctypes.c_double, ctypes.c_double,
                                       ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_float,
                                       ctypes.c_int64, ctypes.c_int64]
        L.orc_voxelize_get.restype = ctypes.c_int64
        L.orc_voxelize_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int64]
        L.orc_voxelize_free.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def splats_struct(d):
    s = OrcSplats(d.count, _ptr(d.positions), _ptr(d.rotations), _ptr(d.logScales), _ptr(d.opacityLogits),
                  _ptr(d.colorsDC), _ptr(d.colorsSH), d.shBands)
    s._keep = d
    return s


def camera_struct(c):
    cs = OrcCamera()
    cs.width, cs.height = int(c.width), int(c.height)
    for i in range(16):
        cs.view[i] = float(c.viewMatrix[i])
    cs.fov_y, cs.near_plane, cs.far_plane = float(c.fovY), float(c.near), float(c.far)
    cs.projection = 0 if c.projection == "pinhole" else 1
    return cs


_RENDER_DTYPES = {"rgba": np.uint32, "accum": np.float32, "accum64": np.float64, "sorted_idx": np.uint32,
                  "depth_keys": np.uint32, "records": np.float32, "counts": np.uint32, "offsets": np.uint32,
                  "tile_list_off": np.uint32, "tile_list_val": np.uint32, "chunk_tile_offsets": np.uint32,
                  "tile_examined": np.uint32, "tile_evaluated": np.uint32, "n_visible": np.uint64,
                  "n_pairs": np.uint64}

_VOX_DTYPES = {"block_idx": np.uint32, "mask_lo": np.uint32, "mask_hi": np.uint32, "near_idx": np.uint32,
               "near_lo": np.uint32, "near_hi": np.uint32, "near_solid_lo": np.uint32,
               "near_solid_hi": np.uint32, "extents": np.float32, "bounds": np.float64, "dims": np.float64,
               "near_bits": np.uint64, "evals": np.uint64}


def _fetch(getter, h, name, dtype):
    n = getter(h, name.encode(), None, 0)
    if n < 0:
        raise KeyError(name)
    out = np.empty(n // np.dtype(dtype).itemsize, dtype)
    if n:
        getter(h, name.encode(), out.ctypes.data, n)
    return out


def render(data, camera, background=(0.0, 0.0, 0.0, 1.0), maxCoverage=16384, chunkCap=200_000,
           f64=False, fields=("rgba",)):
    """Run the oracle render; returns a dict of the requested fields."""
    L = lib()
    bg = (ctypes.c_float * 4)(*background)
    h = L.orc_render_run(ctypes.byref(splats_struct(data)), ctypes.byref(camera_struct(camera)),
                         maxCoverage, chunkCap, bg, 1 if f64 else 0)
    try:
        out = {f: _fetch(L.orc_render_get, h, f, _RENDER_DTYPES[f]) for f in fields}
    finally:
        L.orc_render_free(h)
    for k in ("n_visible", "n_pairs"):
        if k in out:
            out[k] = int(out[k][0])
    if "rgba" in out:
        out["rgba"] = out["rgba"].view(np.uint8).copy()
    return out


def voxelize(data, voxelResolution=0.05, opacityCutoff=0.1, bounds=None, order=0, eps=1e-5,
             fields=("block_idx", "mask_lo", "mask_hi", "bounds", "dims"), z_rows=None):
    """Run the oracle voxelizer.  order 0: canonical summation order (ascending
    Gaussian index), order 1: the reference's BVH query order.  z_rows=(lo, hi)
    restricts the run to the 16^3-block batches whose z row is in [lo, hi)."""
    L = lib()
    zlo, zhi = (0, 0) if z_rows is None else (int(z_rows[0]), int(z_rows[1]))
    b = None
    if bounds is not None:
        b = (ctypes.c_double * 6)(*[float(v) for v in list(bounds[0]) + list(bounds[1])])
    h = L.orc_voxelize_run(ctypes.byref(splats_struct(data)), voxelResolution, opacityCutoff, b, order, eps,
                           zlo, zhi)
    try:
        out = {f: _fetch(L.orc_voxelize_get, h, f, _VOX_DTYPES[f]) for f in fields}
    finally:
        L.orc_voxelize_free(h)
    for k in ("near_bits", "evals"):
        if k in out:
            out[k] = int(out[k][0])
    return out


def math(op: str, x, y=None):
    """Evaluate a dl_math.h function elementwise (test helper)."""
    L = lib()
    code = {"expf": 0, "atan2f": 1, "asinf": 2, "sortable": 3, "exp": 4}[op]
    if op == "exp":
        x = np.ascontiguousarray(x, np.float64)
        out = np.empty_like(x)
    else:
        x = np.ascontiguousarray(x, np.float32)
        out = np.empty(x.shape, np.uint32 if op == "sortable" else np.float32)
    yy = None if y is None else np.ascontiguousarray(y, np.float32)
    L.orc_math.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
    L.orc_math(code, x.ctypes.data, None if yy is None else yy.ctypes.data, out.ctypes.data, x.size)
    return out
