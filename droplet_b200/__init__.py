"""droplet_b200 — B200-native (sm_100a) forward renderer and voxelizer for
droplet scenes, behind droplet's public API (src/index.ts:16-38)."""
from .types import (BackgroundRGBA, Bounds, RenderCamera, SplatData, mat4Identity, mat4LookAt,
                    numSHCoeffsPerChannel, quatRotate, splatInputStride, vec3)
from ._lib import DropletError
from .ply import loadPlySplats, splatBounds
from .api import (BlockMaskBuffer, Device, GpuRadixSorter, Mlp, PlySplats, Renderer, Scene, VoxelBlock,
                  VoxelizeResult, createDevice, mortonDecode3, mortonEncode3, voxelize, voxelQuery, voxelCarve)

__all__ = ["BackgroundRGBA", "Bounds", "RenderCamera", "SplatData", "mat4Identity", "mat4LookAt",
           "numSHCoeffsPerChannel", "quatRotate", "splatInputStride", "vec3", "DropletError",
           "BlockMaskBuffer", "Device", "GpuRadixSorter", "Mlp", "Renderer", "Scene", "VoxelBlock", "VoxelizeResult", "createDevice",
           "mortonDecode3", "mortonEncode3", "voxelize", "voxelQuery", "voxelCarve", "loadPlySplats", "splatBounds", "PlySplats"]
