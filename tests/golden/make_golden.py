"""Generate tests/golden/kat.json: known answers derived in closed form (f64),
independently of the oracle's code, used to pin the oracle.

The reference publishes no numeric golden vectors (its only tests are the
qualitative browser checks in examples/browser/test.ts:114-273), so the
numeric pins are hand derivations of its formulas for cases with closed forms:

  * one isotropic splat at the origin seen head-on (test.ts:45-56,95-103):
    projected conic, radius, opacity and the centre pixel's byte
    (project.ts:128-217, rasterize.ts:62-79, finalize.ts:30-43);
  * the order-preserving depth key (spatial/radix-sort.ts:20-24) of edge values;
  * one isotropic Gaussian voxelized alone: the solid voxel count, from the
    closest-point Mahalanobis distance and the Beer-Lambert threshold
    (voxel/shaders/voxelize.ts:62-140), and its block-aligned bounds
    (voxelize.ts:278-306).
Run: python tests/golden/make_golden.py
"""
import json
import math
import os
import struct

HERE = os.path.dirname(os.path.abspath(__file__))


def f32(x):
    return struct.unpack("<f", struct.pack("<f", x))[0]


def sortable(x):
    u = struct.unpack("<I", struct.pack("<f", x))[0]
    return (~u & 0xFFFFFFFF) if (u & 0x80000000) else (u ^ 0x80000000)


def one_splat():
    W = H = 128
    focal = H / (2 * math.tan(math.pi / 6))
    s = math.exp(-2.5)
    z = 4.0
    c = (focal * s / z) ** 2                   # J Σ Jᵀ diagonal for a head-on isotropic splat
    cb = c + 0.3
    det = cb * cb
    conic = 1.0 / cb
    aa = math.sqrt(c * c / det)
    radius = math.ceil(3.0 * math.sqrt(cb))
    alpha = 1 / (1 + math.exp(-3.0)) * 1.0 * aa
    # centre pixel (64, 64): pixel centre (64.5, 64.5), splat at (64, 64)
    power = -0.5 * (conic * 0.25 + conic * 0.25)
    a = min(0.999, alpha * max(0.0, math.exp(power) - math.exp(-4.5)))
    byte = int(a * 1.0 * 255 + 0.5)            # colour (1,0,0): dc = 0.5 -> 0.5 + 0.5
    tiles = (math.floor((64 + radius) / 16) - math.floor((64 - radius) / 16) + 1) ** 2
    return {"screen": [64.0, 64.0], "radius": radius, "depth": 4.0, "conicA": conic, "conicB": 0.0,
            "conicC": conic, "alpha": alpha, "centre_byte": byte, "tile_count": tiles}


def voxel_single():
    # Gaussian at the origin, isotropic scale 0.1, opacity logit 3, res 0.05, cutoff 0.1
    res, s, cutoff = 0.05, 0.1, 0.1
    op = 1 / (1 + math.exp(-3.0))
    ext = 3 * s
    bs = 4 * res
    bmin = math.floor(-ext / bs) * bs
    bmax = math.ceil(ext / bs) * bs
    dims = round((bmax - bmin) / bs)
    half = res / 2
    n = int(round((bmax - bmin) / res))
    solid = 0
    for i in range(n):
        for j in range(n):
            for k in range(n):
                c = [bmin + (t + 0.5) * res for t in (i, j, k)]
                if any(abs(v) > ext + half for v in c):
                    continue
                cd = [min(max(0.0, v - half), v + half) for v in c]   # closest point to the centre
                d2 = sum(x * x for x in cd) / (s * s)
                sigma = op * math.exp(-0.5 * d2)
                if 1 - math.exp(-sigma) >= cutoff:
                    solid += 1
    return {"bounds_min": bmin, "bounds_max": bmax, "dims": dims, "solid_voxels": solid}


def main():
    keys = {repr(v): sortable(v) for v in (0.0, -0.0, 1.0, -1.0, 2.5, -2.5, float("inf"), float("-inf"),
                                           1e-45, -1e-45, 3.4028234663852886e38)}
    kat = {"one_splat": one_splat(), "sortable_keys": keys, "voxel_single": voxel_single()}
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(kat, f, indent=1, sort_keys=True)
    print(json.dumps(kat, indent=1))


if __name__ == "__main__":
    main()
