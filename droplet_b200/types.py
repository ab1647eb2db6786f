"""Host-side data types mirroring droplet's public TypeScript types.

Reference: src/types.ts:23-82 (SplatData, numSHCoeffsPerChannel,
splatInputStride, Bounds, BackgroundRGBA, Projection, RenderCamera) and
src/math/index.ts:41-80 (mat4LookAt, mat4Identity, vec3, quatRotate).

Arrays are numpy ``float32`` in the same struct-of-arrays layout the
TypeScript ``Float32Array`` fields use; a ``viewMatrix`` is 16 float32 values,
column-major, world -> camera.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Literal, Optional, Sequence

import numpy as np

Projection = Literal["pinhole", "equirect"]


def numSHCoeffsPerChannel(bands: int) -> int:
    """types.ts:35-37 — SH coefficients per colour channel for 0..3 bands."""
    return 0 if bands == 0 else 3 if bands == 1 else 8 if bands == 2 else 15


def splatInputStride(bands: int) -> int:
    """types.ts:49-51 — floats per Gaussian in the packed project record."""
    return 14 + 3 * numSHCoeffsPerChannel(bands)


def _f32(a, n: int, name: str) -> np.ndarray:
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(-1))
    if arr.size != n:
        raise ValueError(f"SplatData.{name}: expected {n} floats, got {arr.size}")
    return arr


@dataclass
class SplatData:
    """types.ts:23-32 — Gaussian splats, struct of arrays, all float32.

    colorsSH, when present, holds per Gaussian the channel-major SH terms
    [R[0..M-1], G[0..M-1], B[0..M-1]] with M = numSHCoeffsPerChannel(shBands).
    """
    count: int
    positions: np.ndarray
    rotations: np.ndarray
    logScales: np.ndarray
    opacityLogits: np.ndarray
    colorsDC: np.ndarray
    colorsSH: Optional[np.ndarray] = None
    shBands: int = 0

    def __post_init__(self):
        n = int(self.count)
        if n < 0:
            raise ValueError("SplatData.count must be >= 0")
        if self.shBands not in (0, 1, 2, 3):
            raise ValueError("SplatData.shBands must be 0, 1, 2 or 3")
        self.count = n
        self.positions = _f32(self.positions, 3 * n, "positions")
        self.rotations = _f32(self.rotations, 4 * n, "rotations")
        self.logScales = _f32(self.logScales, 3 * n, "logScales")
        self.opacityLogits = _f32(self.opacityLogits, n, "opacityLogits")
        self.colorsDC = _f32(self.colorsDC, 3 * n, "colorsDC")
        if self.colorsSH is not None:
            self.colorsSH = _f32(self.colorsSH, 3 * numSHCoeffsPerChannel(self.shBands) * n, "colorsSH")

    @staticmethod
    def empty() -> "SplatData":
        z = np.zeros(0, np.float32)
        return SplatData(0, z, z, z, z, z, None, 0)


@dataclass
class RenderCamera:
    """types.ts:74-82. viewMatrix: world->camera, column-major, 16 floats."""
    width: int
    height: int
    viewMatrix: np.ndarray
    fovY: float
    near: float
    far: float
    projection: Projection = "pinhole"

    def __post_init__(self):
        self.viewMatrix = _f32(self.viewMatrix, 16, "viewMatrix")
        if self.projection not in ("pinhole", "equirect"):
            raise ValueError("RenderCamera.projection must be 'pinhole' or 'equirect'")


@dataclass
class BackgroundRGBA:
    """types.ts:63-68 — background colour in [0, 1]."""
    r: float = 0.0
    g: float = 0.0
    b: float = 0.0
    a: float = 1.0


@dataclass
class Bounds:
    """types.ts:54-57."""
    min: Sequence[float] = field(default_factory=lambda: (0.0, 0.0, 0.0))
    max: Sequence[float] = field(default_factory=lambda: (0.0, 0.0, 0.0))


def vec3(x: float, y: float, z: float):
    return (float(x), float(y), float(z))


def mat4Identity() -> np.ndarray:
    m = np.zeros(16, np.float32)
    m[0] = m[5] = m[10] = m[15] = 1.0
    return m


def _norm(v):
    length = math.hypot(v[0], v[1], v[2])
    return (v[0] / length, v[1] / length, v[2] / length) if length > 0 else (0.0, 0.0, 0.0)


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def mat4LookAt(eye, target, up) -> np.ndarray:
    """math/index.ts:41-56 — right-handed look-at in f64, stored as float32."""
    f = _norm((target[0] - eye[0], target[1] - eye[1], target[2] - eye[2]))
    s = _norm(_cross(f, up))
    u = _cross(s, f)
    m = np.zeros(16, np.float64)
    m[0], m[1], m[2], m[3] = s[0], u[0], -f[0], 0.0
    m[4], m[5], m[6], m[7] = s[1], u[1], -f[1], 0.0
    m[8], m[9], m[10], m[11] = s[2], u[2], -f[2], 0.0
    m[12] = -(s[0] * eye[0] + s[1] * eye[1] + s[2] * eye[2])
    m[13] = -(u[0] * eye[0] + u[1] * eye[1] + u[2] * eye[2])
    m[14] = f[0] * eye[0] + f[1] * eye[1] + f[2] * eye[2]
    m[15] = 1.0
    return m.astype(np.float32)


def quatRotate(q, v):
    """math/index.ts:70-80 — Rodrigues rotation by a [w, x, y, z] quaternion."""
    qw, qx, qy, qz = q
    tx = 2 * (qy * v[2] - qz * v[1])
    ty = 2 * (qz * v[0] - qx * v[2])
    tz = 2 * (qx * v[1] - qy * v[0])
    return (v[0] + qw * tx + (qy * tz - qz * ty),
            v[1] + qw * ty + (qz * tx - qx * tz),
            v[2] + qw * tz + (qx * ty - qy * tx))
