"""Host-side mirror of droplet's public API over the C ABI.

Same names, argument meaning and error behaviour as the TypeScript entry
points (src/index.ts:16-38):

  createDevice(opts)                       src/gpu/device.ts:27-41
  Renderer(device, opts).render(...)       src/render/pipeline.ts:50-592
  voxelize(device, data, opts)             src/voxel/voxelize.ts:59-248
  BlockMaskBuffer                          src/voxel/block-mask-buffer.ts:23-64

Every call goes through libdroplet_b200.so; a non-zero status raises
DropletError (the TypeScript shim throws Error the same way).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence, Union

import numpy as np

from . import _lib
from ._lib import DropletError, check
from .types import BackgroundRGBA, Bounds, RenderCamera, SplatData, numSHCoeffsPerChannel


def _splats(d: SplatData) -> _lib.DlSplats:
    s = _lib.DlSplats()
    s.count = d.count
    p = lambda a: None if a is None or a.size == 0 else a.ctypes.data
    s.positions, s.rotations, s.log_scales = p(d.positions), p(d.rotations), p(d.logScales)
    s.opacity_logits, s.colors_dc, s.colors_sh = p(d.opacityLogits), p(d.colorsDC), p(d.colorsSH)
    s.sh_bands = d.shBands
    s._keep = d
    return s


def _camera(c: RenderCamera) -> _lib.DlCamera:
    cs = _lib.DlCamera()
    cs.width, cs.height = int(c.width), int(c.height)
    ctypes.memmove(cs.view, np.ascontiguousarray(c.viewMatrix, np.float32).ctypes.data, 64)
    cs.fov_y, cs.near_plane, cs.far_plane = float(c.fovY), float(c.near), float(c.far)
    cs.projection = _lib.DL_PINHOLE if (c.projection or "pinhole") == "pinhole" else _lib.DL_EQUIRECT
    return cs


def _bg(bg) -> ctypes.Array:
    if bg is None:
        bg = BackgroundRGBA()
    if isinstance(bg, BackgroundRGBA):
        vals = (bg.r, bg.g, bg.b, bg.a)
    elif isinstance(bg, dict):
        vals = (bg["r"], bg["g"], bg["b"], bg["a"])
    else:
        vals = tuple(bg)
    return (ctypes.c_float * 4)(*[float(v) for v in vals])


class Device:
    """Opaque handle standing in for GPUDevice (one CUDA device + stream)."""

    def __init__(self, handle: int, ordinal: int):
        self._h = handle
        self.ordinal = ordinal

    @property
    def handle(self):
        if not self._h:
            raise DropletError(_lib.DL_E_INVALID_ARG, "device is closed")
        return self._h

    def set_voxel_scheduler(self, mlp: Optional["Mlp"]):
        """Attach (or with None detach) the block-cost model that orders voxelize's
        block queue on this device; the order changes timing only."""
        check(_lib.load().dl_device_set_voxel_scheduler(self.handle, mlp.handle if mlp is not None else None))
        self._vox_sched = mlp

    def destroy(self):
        if self._h:
            _lib.load().dl_device_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def createDevice(opts: Optional[dict] = None) -> Device:
    """device.ts:27-41.  opts: {"device": Device} passes an existing device
    through; {"ordinal": k} picks a CUDA device.  Raises if none is usable."""
    opts = opts or {}
    if opts.get("device") is not None:
        return opts["device"]
    L = _lib.load()
    h = ctypes.c_void_p()
    ordinal = int(opts.get("ordinal", 0))
    check(L.dl_device_open(ordinal, ctypes.byref(h)))
    return Device(h.value, ordinal)


class Scene:
    """A device-resident copy of a SplatData (no reference counterpart)."""

    def __init__(self, renderer: "Renderer", handle: int, count: int):
        self._r = renderer
        self._h = handle
        self.count = count

    def destroy(self):
        if self._h:
            _lib.load().dl_scene_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Renderer:
    """pipeline.ts:50-592.  opts: {chunkCap, maxCoveragePerSplat}."""

    STAGES = ("project", "depth_sort", "emit", "tile_offsets", "pair_sort", "rasterize")

    def __init__(self, device: Device, opts: Optional[dict] = None, **kw):
        opts = dict(opts or {}, **kw)
        o = _lib.DlRendererOpts(int(opts.get("chunkCap") or 0), int(opts.get("maxCoveragePerSplat") or 0))
        h = ctypes.c_void_p()
        check(_lib.load().dl_renderer_create(device.handle, ctypes.byref(o), ctypes.byref(h)))
        self._h = h.value
        self.device = device

    @property
    def handle(self):
        if not self._h:
            raise DropletError(_lib.DL_E_INVALID_ARG, "renderer is destroyed")
        return self._h

    def render(self, data: SplatData, camera: RenderCamera, background=None) -> np.ndarray:
        """pipeline.ts:181-426 — returns a fresh uint8 array of width*height*4 (RGBA8)."""
        out = np.empty(int(camera.width) * int(camera.height) * 4, np.uint8)
        check(_lib.load().dl_render(self.handle, ctypes.byref(_splats(data)), ctypes.byref(_camera(camera)),
                                    _bg(background), out.ctypes.data if out.size else None, out.size))
        return out

    def render_many(self, data: SplatData, cameras: Sequence[RenderCamera], background=None, flags: int = 0,
                    outs: Optional[Sequence[int]] = None) -> Optional[List[np.ndarray]]:
        """render() for several cameras of one SplatData in one call (one upload,
        one batched frame).  outs: optional host pointers (e.g. pinned buffers)."""
        n = len(cameras)
        cams = (_lib.DlCamera * n)(*[_camera(c) for c in cameras])
        ptrs = (ctypes.c_void_p * n)()
        host = None
        if outs is None:
            host = [np.empty(int(c.width) * int(c.height) * 4, np.uint8) for c in cameras]
            outs = [a.ctypes.data for a in host]
        for k, p in enumerate(outs):
            ptrs[k] = int(p)
        check(_lib.load().dl_render_many(self.handle, ctypes.byref(_splats(data)), cams, n, _bg(background), ptrs,
                                         flags))
        return host

    # ---- device-resident scenes and batches
    def upload(self, data: SplatData, precision: str = "f32") -> Scene:
        prec = {"f32": _lib.DL_PREC_F32, "f16": _lib.DL_PREC_F16, "bf16": _lib.DL_PREC_BF16}[precision]
        h = ctypes.c_void_p()
        check(_lib.load().dl_scene_upload(self.handle, ctypes.byref(_splats(data)), prec, ctypes.byref(h)))
        return Scene(self, h.value, data.count)

    def render_batch(self, scene: Scene, cameras: Sequence[RenderCamera], background=None, flags: int = 0,
                     outs: Optional[Sequence[int]] = None) -> Optional[List[np.ndarray]]:
        """Render len(cameras) views.  With outs (device pointers) the images stay
        on the device (flag DL_BATCH_OUT_DEVICE is added); otherwise returns a list
        of uint8 arrays."""
        n = len(cameras)
        cams = (_lib.DlCamera * n)(*[_camera(c) for c in cameras])
        ptrs = (ctypes.c_void_p * n)()
        host = None
        if outs is None:
            host = [np.empty(int(c.width) * int(c.height) * 4, np.uint8) for c in cameras]
            for k, a in enumerate(host):
                ptrs[k] = a.ctypes.data
        else:
            flags |= _lib.DL_BATCH_OUT_DEVICE
            for k, p in enumerate(outs):
                ptrs[k] = int(p)
        check(_lib.load().dl_render_batch(self.handle, scene._h, cams, n, _bg(background), ptrs, flags))
        return host

    RASTER_SHAPES = ("8x4", "16x2", "4x8", "8x8x2", "8x4-f32x2", "tile-f32x2", "tile")

    BIN_TILES = ("16x16", "8x8", "32x8")

    def set_tuning(self, pair_sort_bits: int = 8, raster_shape: str = "tile-f32x2", raster_ctas_per_sm: int = 0,
                   bin_tile: str = "16x16"):
        """Timing-only knobs of rendered frames (dl_tuning); no knob changes a pixel."""
        t = _lib.DlTuning(int(pair_sort_bits), self.RASTER_SHAPES.index(raster_shape), int(raster_ctas_per_sm),
                          self.BIN_TILES.index(bin_tile))
        check(_lib.load().dl_renderer_set_tuning(self.handle, ctypes.byref(t)))

    def get_tuning(self) -> dict:
        t = _lib.DlTuning()
        check(_lib.load().dl_renderer_get_tuning(self.handle, ctypes.byref(t)))
        return {"pair_sort_bits": t.pair_sort_bits, "raster_shape": self.RASTER_SHAPES[t.raster_shape],
                "raster_ctas_per_sm": t.raster_ctas_per_sm, "bin_tile": self.BIN_TILES[t.bin_tile]}

    def autotune(self, scene: Scene, cameras: Sequence[RenderCamera], background=None, flags: int = 0,
                 reps: int = 3) -> dict:
        """Pick the fastest tuning for this batch (coordinate descent over the
        knobs, each candidate timed on the device) and keep it on the renderer."""
        cams = (_lib.DlCamera * len(cameras))(*[_camera(c) for c in cameras])
        best = _lib.DlTuning()
        ms = ctypes.c_double()
        check(_lib.load().dl_renderer_autotune(self.handle, scene._h, cams, len(cameras), _bg(background), flags,
                                               reps, ctypes.byref(best), ctypes.byref(ms)))
        out = self.get_tuning()
        out["frame_ms"] = float(ms.value)
        return out

    def set_scheduler(self, mlp: Optional["Mlp"]):
        """Attach the learned tile-cost model (batched frames then rasterize
        tiles longest-predicted first); None restores launch order."""
        self._sched = mlp
        check(_lib.load().dl_renderer_set_scheduler(self.handle, mlp.handle if mlp else None))

    def tile_log(self):
        """(features [T, 12], measured cost [T]) of the last frame rendered with
        DL_BATCH_LOG_TILES."""
        L = _lib.load()
        n = ctypes.c_uint64()
        check(L.dl_renderer_tile_log(self.handle, None, None, 0, ctypes.byref(n)))
        T = int(n.value)
        feats = np.empty((T, _lib.DL_MLP_IN), np.float32)
        cost = np.empty(T, np.float32)
        if T:
            check(L.dl_renderer_tile_log(self.handle, feats.ctypes.data, cost.ctypes.data, T, ctypes.byref(n)))
        return feats, cost

    # ---- instrumentation
    def set_stream(self, stream_ptr: Optional[int]):
        check(_lib.load().dl_renderer_set_stream(self.handle, stream_ptr))

    def set_debug(self, on: bool = True):
        check(_lib.load().dl_renderer_set_debug(self.handle, 1 if on else 0))

    def set_profiling(self, on: bool = True):
        check(_lib.load().dl_renderer_set_profiling(self.handle, 1 if on else 0))

    def stage_times(self) -> dict:
        ms = (ctypes.c_double * 6)()
        check(_lib.load().dl_renderer_stage_times(self.handle, ms, 6))
        return dict(zip(self.STAGES, list(ms)))

    def launch_count(self) -> int:
        c = ctypes.c_uint64()
        check(_lib.load().dl_renderer_launch_count(self.handle, ctypes.byref(c)))
        return int(c.value)

    def debug_get(self, name: str, dtype) -> np.ndarray:
        L = _lib.load()
        n = ctypes.c_size_t()
        check(L.dl_renderer_debug_get(self.handle, name.encode(), None, 0, ctypes.byref(n)))
        out = np.empty(n.value // np.dtype(dtype).itemsize, dtype)
        if n.value:
            check(L.dl_renderer_debug_get(self.handle, name.encode(), out.ctypes.data, n.value, ctypes.byref(n)))
        return out

    def destroy(self):
        """pipeline.ts:581-591."""
        if self._h:
            _lib.load().dl_renderer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


# ---------------------------------------------------------------- PLY through the C ABI
class PlySplats:
    """A PLY file parsed by the library (dl_ply_load, src/io/ply.ts:120-239)
    into arrays it owns — page-locked with pinned=True, so rendering or
    uploading them needs no staging copy.  .data is a SplatData whose arrays
    view that memory (valid until destroy())."""

    def __init__(self, source: Union[bytes, bytearray, memoryview, str], opts: Optional[dict] = None,
                 pinned: bool = False):
        if isinstance(source, str):
            with open(source, "rb") as f:
                source = f.read()
        buf = bytes(source)
        flip = True if not opts or opts.get("flipY") is None else bool(opts["flipY"])
        L = _lib.load()
        h = ctypes.c_void_p()
        st = L.dl_ply_load(buf, len(buf), 1 if flip else 0, _lib.DL_PLY_PINNED if pinned else 0, ctypes.byref(h))
        if st != _lib.DL_OK:
            msg = L.dl_last_error().decode(errors="replace")
            if st == _lib.DL_E_INVALID_ARG:
                raise ValueError(msg)            # the reference throws Error with the same message
            raise DropletError(st, msg)
        self._h = h.value
        s = _lib.DlSplats()
        check(L.dl_ply_splats(self._h, ctypes.byref(s)))
        n = int(s.count)

        def view(ptr, k):
            if not ptr or k == 0:
                return None
            buf = (ctypes.c_float * k).from_address(ptr)
            buf._owner = self                    # the arrays keep the parsed memory alive
            return np.frombuffer(buf, dtype=np.float32)
        self.data = SplatData(n, view(s.positions, 3 * n), view(s.rotations, 4 * n), view(s.log_scales, 3 * n),
                              view(s.opacity_logits, n), view(s.colors_dc, 3 * n),
                              view(s.colors_sh, 3 * numSHCoeffsPerChannel(s.sh_bands) * n) if s.sh_bands else None,
                              int(s.sh_bands))

    def destroy(self):
        if self._h:
            _lib.load().dl_ply_free(self._h)
            self._h = None
            self.data = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


# ---------------------------------------------------------------- voxelize
@dataclass
class VoxelBlock:
    """block-mask-buffer.ts:14-21."""
    blockIdx: int
    maskLo: int
    maskHi: int


def _popcount32(a: np.ndarray) -> int:
    """block-mask-buffer.ts:60-64 (SWAR popcount), summed over an array."""
    v = a.astype(np.uint64)
    v = v - ((v >> 1) & 0x55555555)
    v = (v & 0x33333333) + ((v >> 2) & 0x33333333)
    v = (((v + (v >> 4)) & 0x0F0F0F0F) * 0x01010101) & 0xFFFFFFFF
    return int(np.sum(v >> 24))


class BlockMaskBuffer:
    """block-mask-buffer.ts:23-58: sparse 4x4x4-voxel blocks, 2 x u32 masks each,
    in insertion order; the masks are kept as numpy columns."""

    def __init__(self, blockIdx=None, maskLo=None, maskHi=None):
        self.blockIdx = np.asarray(blockIdx if blockIdx is not None else [], np.uint32)
        self.maskLo = np.asarray(maskLo if maskLo is not None else [], np.uint32)
        self.maskHi = np.asarray(maskHi if maskHi is not None else [], np.uint32)
        self._index = None

    def _map(self):
        if self._index is None:
            self._index = {int(b): i for i, b in enumerate(self.blockIdx.tolist())}
        return self._index

    def addBlock(self, blockIdx: int, maskLo: int, maskHi: int) -> None:
        if maskLo == 0 and maskHi == 0:
            return
        m = self._map()
        i = m.get(int(blockIdx))
        if i is None:
            m[int(blockIdx)] = len(self.blockIdx)
            self.blockIdx = np.append(self.blockIdx, np.uint32(blockIdx))
            self.maskLo = np.append(self.maskLo, np.uint32(maskLo))
            self.maskHi = np.append(self.maskHi, np.uint32(maskHi))
        else:
            self.maskLo[i] |= np.uint32(maskLo)
            self.maskHi[i] |= np.uint32(maskHi)

    def get(self, blockIdx: int) -> Optional[VoxelBlock]:
        i = self._map().get(int(blockIdx))
        if i is None:
            return None
        return VoxelBlock(int(self.blockIdx[i]), int(self.maskLo[i]), int(self.maskHi[i]))

    @property
    def blocks(self) -> List[VoxelBlock]:
        return [VoxelBlock(int(b), int(lo), int(hi)) for b, lo, hi in zip(self.blockIdx, self.maskLo, self.maskHi)]

    def popcount(self) -> int:
        return _popcount32(self.maskLo) + _popcount32(self.maskHi)

    @property
    def count(self) -> int:
        return int(self.blockIdx.size)


@dataclass
class VoxelizeResult:
    """voxelize.ts:38-45."""
    buffer: BlockMaskBuffer
    bounds: Bounds
    voxelResolution: float
    numBlocksX: float
    numBlocksY: float
    numBlocksZ: float
    blockLog: Optional[tuple] = None           # (features [n, 12], cost [n]) with opts["logBlocks"]
    stageTimes: Optional[dict] = None          # device ms per stage with opts["profile"]


def voxelQuery(device: Device, result: VoxelizeResult, points) -> np.ndarray:
    """Occupancy of points (n x 3 float32) against a voxelize result, on the device
    (dl_vox_query; no counterpart in the reference, whose BlockMaskBuffer.get
    answers one block at a time on the CPU).  Returns n uint8: 1 where the
    point's voxel floor((p - bounds.min) / voxelResolution) is solid."""
    pts = np.ascontiguousarray(np.asarray(points, np.float32).reshape(-1, 3))
    out = np.zeros(len(pts), np.uint8)
    buf = result.buffer
    idx = np.ascontiguousarray(buf.blockIdx, np.uint32)
    lo = np.ascontiguousarray(buf.maskLo, np.uint32)
    hi = np.ascontiguousarray(buf.maskHi, np.uint32)
    bmin = (ctypes.c_double * 3)(*[float(x) for x in result.bounds.min])
    dims = (ctypes.c_double * 3)(float(result.numBlocksX), float(result.numBlocksY), float(result.numBlocksZ))
    check(_lib.load().dl_vox_query(device.handle, idx.ctypes.data, lo.ctypes.data, hi.ctypes.data, len(idx), bmin,
                                   float(result.voxelResolution), dims, pts.ctypes.data, len(pts), out.ctypes.data))
    return out


def voxelCarve(device: Device, a: BlockMaskBuffer, b: BlockMaskBuffer) -> BlockMaskBuffer:
    """A minus B, block by block, on the device (dl_vox_carve; voxelize.ts:1-14
    names carve among the buffer's downstream stages, which the reference does not
    build).  Each of A's blocks keeps the bits B's blocks with the same index do
    not set; blocks left empty are dropped, the rest keep A's order."""
    cols = []
    for buf in (a, b):
        cols.append([np.ascontiguousarray(c, np.uint32) for c in (buf.blockIdx, buf.maskLo, buf.maskHi)])
    (ai, al, ah), (bi, bl, bh) = cols
    na = len(ai)
    oi, ol, oh = (np.zeros(max(na, 1), np.uint32) for _ in range(3))
    n = ctypes.c_uint64(0)
    check(_lib.load().dl_vox_carve(device.handle, ai.ctypes.data, al.ctypes.data, ah.ctypes.data, na,
                                   bi.ctypes.data, bl.ctypes.data, bh.ctypes.data, len(bi),
                                   oi.ctypes.data, ol.ctypes.data, oh.ctypes.data, ctypes.byref(n)))
    k = n.value
    return BlockMaskBuffer(oi[:k].copy(), ol[:k].copy(), oh[:k].copy())


def voxelize(device: Device, data: SplatData, opts: Optional[dict] = None) -> VoxelizeResult:
    """voxelize.ts:59-248.  opts: {voxelResolution=0.05, opacityCutoff=0.1, bounds}.

    opts["shard"] = (index, count) voxelizes only that shard of the grid's z rows
    of 16^3-block batches (see droplet_b200.shard); bounds and numBlocks stay
    those of the whole grid.  opts["fastExp"] evaluates the densities with the
    hardware ex2 (bits within about 1e-5 of the cutoff may change)."""
    opts = opts or {}
    o = _lib.DlVoxOpts()
    res = opts.get("voxelResolution")
    cut = opts.get("opacityCutoff")
    o.voxel_resolution = 0.05 if res is None else float(res)
    o.opacity_cutoff = 0.1 if cut is None else float(cut)
    o.use_defaults = 0
    b = opts.get("bounds")
    if b is not None:
        bmin, bmax = (b.min, b.max) if isinstance(b, Bounds) else (b["min"], b["max"])
        o.has_bounds = 1
        for k in range(3):
            o.bounds_min[k] = float(bmin[k])
            o.bounds_max[k] = float(bmax[k])
    sh = opts.get("shard")
    if sh is not None:
        o.shard_index, o.shard_count = int(sh[0]), int(sh[1])
    o.log_blocks = 1 if opts.get("logBlocks") else 0
    o.flags = (_lib.DL_VOX_FAST_EXP if opts.get("fastExp") else 0) | (_lib.DL_VOX_PROFILE if opts.get("profile") else 0)
    L = _lib.load()
    h = ctypes.c_void_p()
    check(L.dl_voxelize(device.handle, ctypes.byref(_splats(data)), ctypes.byref(o), ctypes.byref(h)))
    try:
        bmin = (ctypes.c_double * 3)()
        bmax = (ctypes.c_double * 3)()
        dims = (ctypes.c_double * 3)()
        cnt = ctypes.c_uint64()
        check(L.dl_vox_result_info(h, bmin, bmax, dims, ctypes.byref(cnt)))
        n = int(cnt.value)
        idx = np.empty(n, np.uint32)
        lo = np.empty(n, np.uint32)
        hi = np.empty(n, np.uint32)
        if n:
            check(L.dl_vox_result_copy(h, idx.ctypes.data, lo.ctypes.data, hi.ctypes.data))
        stages = None
        if opts.get("profile"):
            ms = (ctypes.c_double * 7)()
            check(L.dl_vox_result_stage_times(h, ms, 7))
            stages = dict(zip(("prep", "binning", "sort", "heads", "eval", "compact", "host"), list(ms)))
        log = None
        if o.log_blocks:
            m = ctypes.c_uint64()
            check(L.dl_vox_result_block_log(h, None, None, 0, ctypes.byref(m)))
            f = np.empty((int(m.value), _lib.DL_MLP_IN), np.float32)
            c = np.empty(int(m.value), np.float32)
            if m.value:
                check(L.dl_vox_result_block_log(h, f.ctypes.data, c.ctypes.data, m.value, ctypes.byref(m)))
            log = (f, c)
    finally:
        L.dl_vox_result_free(h)
    return VoxelizeResult(BlockMaskBuffer(idx, lo, hi), Bounds(tuple(bmin), tuple(bmax)),
                          o.voxel_resolution, dims[0], dims[1], dims[2], log, stages)


# ---------------------------------------------------------------- learned tile-cost model
class Mlp:
    """The renderer's tile-cost model (12 -> 64 -> 64 -> 1, BF16 weights), trained
    and evaluated by the library's own kernels."""

    def __init__(self, device: Device, seed: int = 0):
        h = ctypes.c_void_p()
        check(_lib.load().dl_mlp_create(device.handle, seed, ctypes.byref(h)))
        self._h = h.value
        self.device = device

    @property
    def handle(self):
        if not self._h:
            raise DropletError(_lib.DL_E_INVALID_ARG, "model is destroyed")
        return self._h

    def get_params(self) -> np.ndarray:
        p = np.empty(_lib.DL_MLP_PARAMS, np.float32)
        check(_lib.load().dl_mlp_get_params(self.handle, p.ctypes.data, p.size))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        check(_lib.load().dl_mlp_set_params(self.handle, p.ctypes.data, p.size))

    def predict(self, X) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32).reshape(-1, _lib.DL_MLP_IN)
        out = np.empty(len(X), np.float32)
        check(_lib.load().dl_mlp_predict(self.handle, X.ctypes.data, len(X), out.ctypes.data))
        return out

    def grad(self, X, y):
        X = np.ascontiguousarray(X, np.float32).reshape(-1, _lib.DL_MLP_IN)
        y = np.ascontiguousarray(y, np.float32)
        g = np.empty(_lib.DL_MLP_PARAMS, np.float32)
        loss = ctypes.c_float()
        check(_lib.load().dl_mlp_grad(self.handle, X.ctypes.data, y.ctypes.data, len(X), g.ctypes.data,
                                      ctypes.byref(loss)))
        return g, float(loss.value)

    def train(self, X, y, epochs=10, batch=4096, lr=1e-3, seed=0) -> float:
        X = np.ascontiguousarray(X, np.float32).reshape(-1, _lib.DL_MLP_IN)
        y = np.ascontiguousarray(y, np.float32)
        loss = ctypes.c_float()
        check(_lib.load().dl_mlp_train(self.handle, X.ctypes.data, y.ctypes.data, len(X), epochs, batch, lr, seed,
                                       ctypes.byref(loss)))
        return float(loss.value)

    def destroy(self):
        if self._h:
            _lib.load().dl_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


# ---------------------------------------------------------------- Morton order (src/voxel/morton.ts:11-22)
def mortonEncode3(x: int, y: int, z: int) -> int:
    """morton.ts:11-14 — in-block index of (x, y, z) in [0, 4)^3, bits z2 y2 x2 z1 y1 x1."""
    return (((x & 1) << 0) | ((y & 1) << 1) | ((z & 1) << 2)
            | ((x & 2) << 2) | ((y & 2) << 3) | ((z & 2) << 4))


def mortonDecode3(m: int):
    """morton.ts:16-22 — inverse of mortonEncode3."""
    return ((m & 1) | ((m >> 2) & 2), ((m >> 1) & 1) | ((m >> 3) & 2), ((m >> 2) & 1) | ((m >> 4) & 2))


# ---------------------------------------------------------------- GpuRadixSorter (src/gpu/radix-sort.ts:91-216)
class _DeviceArray:
    """A library-owned device array seen through __cuda_array_interface__."""

    def __init__(self, ptr: int, n: int, owner):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (ptr, False), "version": 3}
        self._owner = owner


class GpuRadixSorter:
    """GpuRadixSorter(device).sort(keys, vals, n, keyBits=32) -> (keys, vals).

    keys / vals are CUDA tensors of at least n 32-bit elements (torch.uint32 or
    torch.int32 bit patterns); vals may be None (the values are then the input
    positions).  The sort is stable and runs wholly on the device; the result
    is returned as the pair of arrays that hold it (library-owned arrays come
    back as torch.int32 tensors of the same bit patterns) — the inputs or the
    sorter's pong buffers (valid until the next sort), as in the reference.
    """

    def __init__(self, device: Device):
        h = ctypes.c_void_p()
        check(_lib.load().dl_sorter_create(device.handle, ctypes.byref(h)))
        self._h = h.value
        self.device = device

    @property
    def handle(self):
        if not self._h:
            raise DropletError(_lib.DL_E_INVALID_ARG, "sorter is destroyed")
        return self._h

    def set_stream(self, stream_ptr: Optional[int]):
        check(_lib.load().dl_sorter_set_stream(self.handle, stream_ptr or None))

    def set_digit_bits(self, bits: int):
        check(_lib.load().dl_sorter_set_digit_bits(self.handle, int(bits)))

    def sort(self, keys, vals, n: int, keyBits: int = 32):
        import torch
        for t in (keys, vals):
            if t is not None and (not t.is_cuda or t.element_size() != 4 or not t.is_contiguous() or t.numel() < n):
                raise DropletError(_lib.DL_E_INVALID_ARG, "keys / vals must be contiguous 32-bit CUDA tensors "
                                                           "of at least n elements")
        ok, ov = ctypes.c_void_p(), ctypes.c_void_p()
        check(_lib.load().dl_sorter_sort(self.handle, keys.data_ptr(), None if vals is None else vals.data_ptr(),
                                         int(n), int(keyBits), ctypes.byref(ok), ctypes.byref(ov)))

        def wrap(ptr, like):
            if like is not None and ptr == like.data_ptr():
                return like
            if not ptr:
                return None
            return torch.as_tensor(_DeviceArray(ptr, int(n), self), device=keys.device)
        return wrap(ok.value, keys), wrap(ov.value, vals)

    def destroy(self):
        if self._h:
            _lib.load().dl_sorter_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
