"""CPU tests: the oracle (the C++ restatement of the reference) against the
hand-derived known answers in tests/golden/kat.json and the reference's own
browser checks (examples/browser/test.ts:114-273), plus dl_math.h accuracy."""
import json
import math
import os

import numpy as np
import pytest

from droplet_b200 import synth
from droplet_b200.types import SplatData
from oracle import oracle as O

KAT = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "kat.json")))


def nonblack(rgba):
    p = rgba.reshape(-1, 4)
    return int(((p[:, 0] > 5) | (p[:, 1] > 5) | (p[:, 2] > 5)).sum())


# ---------------------------------------------------------------- dl_math.h
def _ulp_err(got, ref):
    ref32 = ref.astype(np.float32)
    ulp = np.abs(np.nextafter(np.abs(ref32), np.float32(np.inf)).astype(np.float64) - np.abs(ref32).astype(np.float64))
    ulp = np.where(ulp == 0, 2.0 ** -149, ulp)
    return np.abs(got.astype(np.float64) - ref) / ulp


def test_expf_within_one_ulp():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(-103, 88.7, 2_000_000), rng.uniform(-5, 5, 1_000_000),
                        np.linspace(-4.6, -4.4, 100_001)]).astype(np.float32)
    got = O.math("expf", x)
    err = _ulp_err(got, np.exp(x.astype(np.float64)))
    assert err.max() < 1.0, err.max()
    assert O.math("expf", np.array([0.0], np.float32))[0] == 1.0
    assert np.isinf(O.math("expf", np.array([89.0], np.float32))[0])
    assert O.math("expf", np.array([-110.0], np.float32))[0] == 0.0


def test_expf_monotone_below_gaussian_floor():
    # the rasterizer's alpha is exactly 0 whenever exp(power) <= exp(-4.5) (f32 constant);
    # exhaustively: dl_expf is non-decreasing on [-10, -4] (every float in the range)
    lo, hi = np.float32(-10.0).view(np.uint32), np.float32(-4.0).view(np.uint32)
    bits = np.arange(hi, lo + 1, dtype=np.uint32)
    x = bits.view(np.float32)[::-1]          # ascending values
    y = O.math("expf", x)
    assert np.all(np.diff(y.astype(np.float64)) >= 0)


def test_exp_f64_and_inverse_trig():
    rng = np.random.default_rng(1)
    x = rng.uniform(-700, 700, 1_000_000)
    got = O.math("exp", x)
    rel = np.abs(got - np.exp(x)) / np.exp(x)
    assert rel.max() < 3e-16
    y = rng.uniform(-10, 10, 500_000).astype(np.float32)
    z = rng.uniform(-10, 10, 500_000).astype(np.float32)
    a = O.math("atan2f", y, z)
    assert _ulp_err(a, np.arctan2(y.astype(np.float64), z.astype(np.float64))).max() <= 0.5 + 1e-9
    s = rng.uniform(-1, 1, 500_000).astype(np.float32)
    b = O.math("asinf", s)
    assert _ulp_err(b, np.arcsin(s.astype(np.float64))).max() <= 0.5 + 1e-9


def test_sortable_key_edge_values():
    for k, v in KAT["sortable_keys"].items():
        got = int(O.math("sortable", np.array([float(k)], np.float32))[0])
        assert got == v, (k, got, v)
    x = np.sort(np.random.default_rng(2).normal(0, 100, 10000).astype(np.float32))
    keys = O.math("sortable", x)
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)


# ---------------------------------------------------------------- oracle pins
def test_one_splat_closed_form():
    k = KAT["one_splat"]
    r = O.render(synth.one_splat((0, 0, 0)), synth.front_camera(),
                 fields=("rgba", "records", "counts", "n_pairs"))
    rec = r["records"]
    assert rec[0] == k["screen"][0] and rec[1] == k["screen"][1]
    assert rec[2] == k["radius"] and rec[3] == k["depth"]
    assert rec[4] == pytest.approx(k["conicA"], rel=2e-6)
    assert rec[5] == 0.0
    assert rec[6] == pytest.approx(k["conicC"], rel=2e-6)
    assert rec[7] == pytest.approx(k["alpha"], rel=2e-6)
    assert int(r["counts"][0]) == k["tile_count"] == r["n_pairs"]
    img = r["rgba"].reshape(128, 128, 4)
    assert int(img[64, 64, 0]) == k["centre_byte"]
    assert tuple(img[0, 0]) == (0, 0, 0, 255)


def test_voxel_single_closed_form():
    k = KAT["voxel_single"]
    d = SplatData(1, np.zeros(3, np.float32), np.array([1, 0, 0, 0], np.float32),
                  np.full(3, math.log(0.1), np.float32), np.array([3.0], np.float32), np.zeros(3, np.float32))
    v = O.voxelize(d, 0.05, 0.1)
    assert v["bounds"][0] == pytest.approx(k["bounds_min"]) and v["bounds"][3] == pytest.approx(k["bounds_max"])
    assert v["dims"][0] == k["dims"]
    bits = sum(bin(int(a)).count("1") + bin(int(b)).count("1") for a, b in zip(v["mask_lo"], v["mask_hi"]))
    assert bits == k["solid_voxels"]


# ---------------------------------------------------------------- the reference's browser checks
def test_ref_empty_scene_all_black():                          # test.ts:114-124
    r = O.render(SplatData.empty(), synth.front_camera())
    assert nonblack(r["rgba"]) == 0


def test_ref_one_splat_symmetric():                            # test.ts:126-140
    img = O.render(synth.one_splat((0, 0, 0)), synth.front_camera())["rgba"].reshape(128, 128, 4)[..., 0]
    c, l, r, u, d = img[64, 64], img[64, 54], img[64, 74], img[54, 64], img[74, 64]
    assert c > 100 and abs(int(l) - int(r)) < 10 and abs(int(u) - int(d)) < 10


def test_ref_three_splats_rgb():                               # test.ts:142-163
    d = SplatData(3, [0, 0, 1, 0.5, 0, 0.8, -0.5, 0.3, 0.8], [1, 0, 0, 0] * 3, [-2.5] * 9, [3, 3, 3],
                  [0.5, -0.5, -0.5, -0.5, 0.5, -0.5, -0.5, -0.5, 0.5])
    p = O.render(d, synth.front_camera(256, 256))["rgba"].reshape(-1, 4).astype(int)
    r, g, b = p[:, 0], p[:, 1], p[:, 2]
    assert ((r > 50) & (r > g) & (r > b)).sum() > 50
    assert ((g > 50) & (g > r) & (g > b)).sum() > 50
    assert ((b > 50) & (b > r) & (b > g)).sum() > 50


def test_ref_depth_occlusion():                                # test.ts:165-180
    d = SplatData(2, [0, 0, 1, 0, 0, -1], [1, 0, 0, 0] * 2, [-2.5] * 6, [4, 4], [0.5, -0.5, -0.5, -0.5, 0.5, -0.5])
    px = O.render(d, synth.front_camera())["rgba"].reshape(128, 128, 4)[64, 64]
    assert px[0] > 200 and px[1] < 50


def test_ref_sphere_disc():                                    # test.ts:182-190
    nb = nonblack(O.render(synth.many_splats(5000, "sphere"), synth.front_camera(256, 256))["rgba"])
    assert 10000 < nb < 30000


def test_ref_chunk_invariance():                               # test.ts:192-213 (max diff <= 2 there; exact here)
    d = synth.many_splats(200_000, "random")
    a = O.render(d, synth.front_camera(64, 64), fields=("rgba", "accum", "tile_list_val"))
    b = O.render(d, synth.front_camera(64, 64), chunkCap=50_000, fields=("rgba", "accum", "tile_list_val"))
    assert np.array_equal(a["rgba"], b["rgba"])
    assert np.array_equal(a["accum"].view(np.uint32), b["accum"].view(np.uint32))
    assert np.array_equal(a["tile_list_val"], b["tile_list_val"])


def test_ref_large_pairs_dense():                              # test.ts:215-243 (seeded here)
    n = 200_000
    rng = np.random.default_rng(7)
    pos = ((rng.random((n, 3)) - 0.5) * 0.1).astype(np.float32)
    rot = np.zeros((n, 4), np.float32); rot[:, 0] = 1
    dc = np.zeros((n, 3), np.float32); dc[:, 0] = 0.5
    d = SplatData(n, pos, rot, np.full((n, 3), -2.5, np.float32), np.zeros(n, np.float32), dc)
    assert nonblack(O.render(d, synth.front_camera(256, 256))["rgba"]) > 100


def test_ref_voxelize_sphere_nonempty():                       # test.ts:253-260
    v = O.voxelize(synth.many_splats(5000, "sphere"), 0.05, 0.1)
    assert len(v["block_idx"]) > 0


def test_ref_voxelize_empty():                                 # test.ts:262-273
    v = O.voxelize(SplatData.empty(), 0.05, 0.1)
    assert len(v["block_idx"]) == 0
    assert np.isinf(v["bounds"]).all() and np.all(v["dims"] == -np.inf)


def test_voxel_orders_agree_outside_eps_band():
    # canonical (ascending index) vs the reference's BVH order: differences only
    # where |opacity - cutoff| < eps
    d = synth.cluster_scene(20_000, seed=5, clusters=8, extent=1.0, spread=0.3, log_lo=0.01, log_hi=0.1,
                            op_mu=1.0, op_sigma=1.5)
    f = ("block_idx", "mask_lo", "mask_hi", "near_idx", "near_lo", "near_hi")
    a = O.voxelize(d, 0.05, 0.1, order=0, eps=1e-5, fields=f)
    b = O.voxelize(d, 0.05, 0.1, order=1, eps=1e-5, fields=f)
    assert np.array_equal(a["block_idx"], b["block_idx"]) or len(a["block_idx"]) == len(b["block_idx"])
    ma = {int(i): (int(l), int(h)) for i, l, h in zip(a["block_idx"], a["mask_lo"], a["mask_hi"])}
    mb = {int(i): (int(l), int(h)) for i, l, h in zip(b["block_idx"], b["mask_lo"], b["mask_hi"])}
    near = {int(i): (int(l), int(h)) for i, l, h in zip(a["near_idx"], a["near_lo"], a["near_hi"])}
    for k in set(ma) | set(mb):
        x, y, nz = ma.get(k, (0, 0)), mb.get(k, (0, 0)), near.get(k, (0, 0))
        assert ((x[0] ^ y[0]) & ~nz[0]) == 0 and ((x[1] ^ y[1]) & ~nz[1]) == 0


def test_many_splats_lcg_matches_reference_generator():
    # test.ts:64-65: seed = (seed * 1664525 + 1013904223) | 0; ((seed >>> 0) % 10000) / 10000
    d = synth.many_splats(3, "random")
    seed, vals = 1, []
    for _ in range(18):
        seed = (seed * 1664525 + 1013904223) % 2 ** 32
        vals.append((seed % 10000) / 10000)
    assert d.positions[0] == np.float32((vals[0] - 0.5) * 4)
    assert d.colorsDC[0] == np.float32(vals[3] - 0.5)
