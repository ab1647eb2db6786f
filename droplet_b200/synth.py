"""Seeded synthetic scenes and cameras for the benchmark and the parity tests.

No public dataset is involved: every scene is drawn with
``numpy.random.default_rng(seed)`` (PCG64) in a fixed order — cluster centres,
cluster labels, positions, rotations, log-scales, opacity logits, DC colours,
SH coefficients — in float64 and cast once to float32.

Workloads (all sizes as named):
  * ``plain_100k``   100k Gaussians U[-1,1]^3, 1280x720 pinhole, eye (0,0,4).
  * ``voxel_1m``     1M Gaussians in 64 clusters (centres U[-5,5]^3, members
                     N(c, 0.5^2)), voxelResolution 0.05, opacityCutoff 0.1.
  * ``sh3_3m``       3M Gaussians in 256 clusters in [-10,10]^3 (member spread
                     N(c, 0.5^2)), SH bands 3 (45 coefficients N(0, 0.1)),
                     1920x1080 pinhole eye (0,2,12) + 2048x1024 equirect from
                     the origin looking down -z (fovY pi/3).
  * ``ring64``       64 cameras on a ring of radius 12 at height 2 looking at
                     the origin, resolutions cycling 640x360, 1280x720,
                     1920x1080, 2560x1440 (110.6 Mpix per batch), fovY pi/3.
  * ``zipf_10m``     10M Gaussians in 1024 clusters in [-20,20]^3 with cluster
                     weights proportional to k^-1.2, log-scales U[ln .005, ln .2],
                     SH bands 1, voxelResolution 0.02, 16 ring views 1920x1080.
The reference's browser test fixtures (examples/browser/test.ts:45-103) are
reproduced by ``one_splat``, ``many_splats`` and ``front_camera``.
"""
from __future__ import annotations

import math

import numpy as np

from .types import RenderCamera, SplatData, mat4LookAt, numSHCoeffsPerChannel

RING_RESOLUTIONS = [(640, 360), (1280, 720), (1920, 1080), (2560, 1440)]


def _finish(rng, n, positions, log_lo, log_hi, op_mu, op_sigma, bands) -> SplatData:
    q = rng.normal(0.0, 1.0, (n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    ls = rng.uniform(math.log(log_lo), math.log(log_hi), (n, 3))
    op = rng.normal(op_mu, op_sigma, n)
    dc = rng.normal(0.0, 0.5, (n, 3))
    m = numSHCoeffsPerChannel(bands)
    sh = rng.normal(0.0, 0.1, (n, 3 * m)).astype(np.float32) if m else None
    return SplatData(n, positions.astype(np.float32), q.astype(np.float32), ls.astype(np.float32),
                     op.astype(np.float32), dc.astype(np.float32), sh, bands)


def uniform_scene(n: int, seed: int, extent: float = 1.0, log_lo=0.005, log_hi=0.05,
                  op_mu=0.0, op_sigma=2.0, bands=0) -> SplatData:
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-extent, extent, (n, 3))
    return _finish(rng, n, pos, log_lo, log_hi, op_mu, op_sigma, bands)


def cluster_scene(n: int, seed: int, clusters: int, extent: float, spread: float = 0.5,
                  log_lo=0.005, log_hi=0.05, op_mu=0.0, op_sigma=2.0, bands=0,
                  zipf_s: float | None = None) -> SplatData:
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-extent, extent, (clusters, 3))
    if zipf_s is None:
        labels = rng.integers(0, clusters, n)
    else:
        w = np.arange(1, clusters + 1, dtype=np.float64) ** (-zipf_s)
        labels = rng.choice(clusters, size=n, p=w / w.sum())
    pos = centres[labels] + rng.normal(0.0, spread, (n, 3))
    return _finish(rng, n, pos, log_lo, log_hi, op_mu, op_sigma, bands)


def plain_100k(n: int = 100_000) -> SplatData:
    return uniform_scene(n, seed=0)


def voxel_1m(n: int = 1_000_000) -> SplatData:
    return cluster_scene(n, seed=1, clusters=64, extent=5.0, log_lo=0.01, log_hi=0.1,
                         op_mu=1.0, op_sigma=1.5)


def sh3_3m(n: int = 3_000_000, seed: int = 2) -> SplatData:
    return cluster_scene(n, seed=seed, clusters=256, extent=10.0, bands=3)


def zipf_10m(n: int = 10_000_000) -> SplatData:
    return cluster_scene(n, seed=11, clusters=1024, extent=20.0, log_lo=0.005, log_hi=0.2,
                         bands=1, zipf_s=1.2)


def pinhole(width, height, eye, target=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0), fovY=math.pi / 3,
            near=0.01, far=1000.0) -> RenderCamera:
    return RenderCamera(width, height, mat4LookAt(eye, target, up), fovY, near, far, "pinhole")


def plain_100k_camera() -> RenderCamera:
    return pinhole(1280, 720, (0.0, 0.0, 4.0))


def sh3_3m_cameras():
    return [pinhole(1920, 1080, (0.0, 2.0, 12.0)),
            RenderCamera(2048, 1024, mat4LookAt((0.0, 0.0, 0.0), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0)),
                         math.pi / 3, 0.01, 1000.0, "equirect")]


def zipf_10m_cameras(count: int = 16):
    """16 1920x1080 views of the 10M-Gaussian Zipf scene from a ring around it."""
    return ring_cameras(count, radius=45.0, height=5.0, resolutions=[(1920, 1080)])


def ring_cameras(count: int = 64, radius: float = 12.0, height: float = 2.0, resolutions=None, phase: float = 0.0):
    """Cameras at angle 2*pi*(k + phase)/count on a ring, looking at the origin."""
    res = resolutions or RING_RESOLUTIONS
    cams = []
    for k in range(count):
        a = 2.0 * math.pi * (k + phase) / count
        w, h = res[k % len(res)]
        cams.append(pinhole(w, h, (radius * math.sin(a), height, radius * math.cos(a))))
    return cams


# ---- the reference's browser-test fixtures (examples/browser/test.ts:45-103)

def one_splat(pos, color=(1.0, 0.0, 0.0), logScale=-2.5, opLogit=3.0) -> SplatData:
    return SplatData(1, np.array(pos, np.float32), np.array([1, 0, 0, 0], np.float32),
                     np.full(3, logScale, np.float32), np.array([opLogit], np.float32),
                     np.array([c - 0.5 for c in color], np.float32), None, 0)


def many_splats(n: int, layout: str = "sphere") -> SplatData:
    """test.ts:58-93, including its LCG (seed = seed*1664525 + 1013904223 mod 2^32)."""
    pos = np.zeros((n, 3), np.float64)
    dc = np.zeros((n, 3), np.float64)
    seed = 1

    def rand():
        nonlocal seed
        seed = (seed * 1664525 + 1013904223) & 0xFFFFFFFF
        return (seed % 10000) / 10000

    for i in range(n):
        if layout == "sphere":
            t = i / n
            phi = math.acos(1 - 2 * t)
            theta = math.pi * (1 + math.sqrt(5)) * i
            pos[i] = (math.cos(theta) * math.sin(phi), math.sin(theta) * math.sin(phi), math.cos(phi))
        elif layout == "random":
            pos[i] = ((rand() - 0.5) * 4, (rand() - 0.5) * 4, (rand() - 0.5) * 4)
        else:
            pos[i] = (0.0, 0.0, (i / n) * 2 - 1)
        dc[i] = (rand() - 0.5, rand() - 0.5, rand() - 0.5)
    rot = np.zeros((n, 4), np.float32)
    rot[:, 0] = 1
    return SplatData(n, pos.astype(np.float32), rot, np.full((n, 3), -3.2, np.float32),
                     np.full(n, 2.5, np.float32), dc.astype(np.float32), None, 0)


def front_camera(w=128, h=128) -> RenderCamera:
    """test.ts:95-103 renderFront camera."""
    return pinhole(w, h, (0.0, 0.0, 4.0))
