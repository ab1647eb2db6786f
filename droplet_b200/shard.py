"""Multi-GPU sharding of the render and voxelize paths: one process per GPU.

Both paths split into independent units, so no collective is needed on the
data path (views of a scene are independent; the voxel grid splits into z rows
of 16^3-block batches, and the reference appends blocks in batch order with z
outermost, voxel/voxelize.ts:186-188, so row ranges concatenate in order).

  views_of_rank(n, rank, world)        round-robin view assignment
  render_views_sharded(...)            this rank's views of a resident scene
  voxelize_sharded(...)                this rank's z-row shard of the grid
  gather_images / gather_blocks        results to one rank, in the global order

The gathers use torch.distributed (gloo on CPU tensors, NCCL on CUDA tensors)
and run only when the caller asks for the results on one rank.
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import numpy as np

from .api import BlockMaskBuffer, Device, Renderer, Scene, VoxelizeResult, voxelize
from .types import RenderCamera, SplatData


def views_of_rank(n_views: int, rank: int, world: int) -> List[int]:
    """Indices of the views rank `rank` of `world` renders (round robin)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    return list(range(rank, n_views, world))


def render_views_sharded(renderer: Renderer, scene: Scene, cameras: Sequence[RenderCamera], rank: int, world: int,
                         background=None, flags: int = 0):
    """Render this rank's share of `cameras` (one batched call); returns
    (view indices, list of RGBA8 arrays)."""
    ids = views_of_rank(len(cameras), rank, world)
    if not ids:
        return ids, []
    return ids, renderer.render_batch(scene, [cameras[i] for i in ids], background, flags)


def voxelize_sharded(device: Device, data: SplatData, opts: Optional[dict], rank: int, world: int) -> VoxelizeResult:
    """This rank's shard of voxelize(device, data, opts): the blocks of its
    contiguous range of z rows (ranges balanced by Gaussian-block pairs)."""
    o = dict(opts or {})
    o["shard"] = (rank, world)
    return voxelize(device, data, o)


def _gather_bytes(payload: np.ndarray, dst: int, group=None, device=None) -> Optional[List[np.ndarray]]:
    """Gather one uint8 array per rank to rank dst (variable lengths)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = device if device is not None else torch.device("cpu")
    n = torch.tensor([payload.size], dtype=torch.int64, device=dev)
    sizes = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(s.item()) for s in sizes]
    cap = max(max(sizes), 1)
    buf = torch.zeros(cap, dtype=torch.uint8, device=dev)
    if payload.size:
        buf[:payload.size] = torch.from_numpy(np.ascontiguousarray(payload)).to(dev)
    outs = [torch.zeros(cap, dtype=torch.uint8, device=dev) for _ in range(world)] if rank == dst else None
    dist.gather(buf, outs, dst=dst, group=group)
    if rank != dst:
        return None
    return [o[:s].cpu().numpy() for o, s in zip(outs, sizes)]


def gather_images(ids: Sequence[int], images: Sequence[np.ndarray], n_views: int, dst: int = 0, group=None,
                  device=None) -> Optional[List[np.ndarray]]:
    """Collect every rank's RGBA8 images on rank dst, in global view order."""
    header = np.asarray([len(ids)] + list(ids) + [im.size for im in images], np.int64).view(np.uint8)
    body = np.concatenate([np.asarray(im, np.uint8).reshape(-1) for im in images]) if images else np.zeros(0, np.uint8)
    parts = _gather_bytes(np.concatenate([header, body]), dst, group, device)
    if parts is None:
        return None
    out: List[Optional[np.ndarray]] = [None] * n_views
    for p in parts:
        k = int(p[:8].view(np.int64)[0])
        meta = p[:8 * (1 + 2 * k)].view(np.int64)
        vids, sizes = meta[1:1 + k], meta[1 + k:1 + 2 * k]
        off = 8 * (1 + 2 * k)
        for v, s in zip(vids, sizes):
            out[int(v)] = p[off:off + int(s)].copy()
            off += int(s)
    if any(o is None for o in out):
        raise RuntimeError("gather_images: some views were rendered by no rank")
    return out


def gather_blocks(local: VoxelizeResult, dst: int = 0, group=None, device=None) -> Optional[VoxelizeResult]:
    """Concatenate every rank's shard (rank order = z-row order) on rank dst."""
    b = local.buffer
    payload = np.concatenate([b.blockIdx.astype(np.uint32), b.maskLo.astype(np.uint32),
                              b.maskHi.astype(np.uint32)]).view(np.uint8)
    parts = _gather_bytes(payload, dst, group, device)
    if parts is None:
        return None
    cols = [p.view(np.uint32).reshape(3, -1) for p in parts]
    idx = np.concatenate([c[0] for c in cols]) if cols else np.zeros(0, np.uint32)
    lo = np.concatenate([c[1] for c in cols]) if cols else np.zeros(0, np.uint32)
    hi = np.concatenate([c[2] for c in cols]) if cols else np.zeros(0, np.uint32)
    return VoxelizeResult(BlockMaskBuffer(idx, lo, hi), local.bounds, local.voxelResolution, local.numBlocksX,
                          local.numBlocksY, local.numBlocksZ)
