"""GPU parity of the voxelizer against the oracle, through the C ABI.

The GPU sums each voxel's density over its batch list in ascending Gaussian
index, exactly like the oracle's canonical order, so block lists and masks are
bit-exact.  Against the reference's own summation order (its BVH's DFS order,
ported in the oracle) bits may differ only where |opacity - cutoff| < eps;
those bits are counted."""
import math

import numpy as np
import pytest

import droplet_b200 as dl
from droplet_b200 import synth
from droplet_b200.types import Bounds, SplatData
from oracle import oracle as O

pytestmark = pytest.mark.gpu
EPS = 1e-5


def run_both(device, d, res=0.05, cut=0.1, bounds=None):
    opts = {"voxelResolution": res, "opacityCutoff": cut}
    if bounds is not None:
        opts["bounds"] = Bounds(bounds[0], bounds[1])
    g = dl.voxelize(device, d, opts)
    o = O.voxelize(d, res, cut, bounds=bounds)
    return g, o


def assert_same(g, o):
    assert np.array_equal(g.buffer.blockIdx, o["block_idx"]), "block list / order differs"
    assert np.array_equal(g.buffer.maskLo, o["mask_lo"]) and np.array_equal(g.buffer.maskHi, o["mask_hi"])
    assert np.allclose(np.r_[g.bounds.min, g.bounds.max], o["bounds"]) and \
        np.array_equal([g.numBlocksX, g.numBlocksY, g.numBlocksZ], o["dims"])


def test_sphere_5000(device):                                   # test.ts:253-260
    g, o = run_both(device, synth.many_splats(5000, "sphere"))
    assert g.buffer.count > 0
    assert_same(g, o)


def test_empty(device):                                         # test.ts:262-273
    g = dl.voxelize(device, SplatData.empty(), {"voxelResolution": 0.05, "opacityCutoff": 0.1})
    assert g.buffer.count == 0 and math.isinf(g.bounds.min[0]) and g.numBlocksX == -math.inf


def test_clustered_100k_exact(device):
    g, o = run_both(device, synth.voxel_1m(100_000))
    assert g.buffer.count > 1000
    assert_same(g, o)


def test_slabbed_grid_matches_one_pass(device, monkeypatch):
    # the grid is processed in z rows of 16^3-block batches bounded by a pair
    # capacity; a tiny capacity forces many slabs and must not change anything
    d = synth.voxel_1m(40_000)
    g1 = dl.voxelize(device, d, {"voxelResolution": 0.04, "opacityCutoff": 0.1})
    monkeypatch.setenv("DL_VOX_SLAB_PAIRS", "20000")
    g2 = dl.voxelize(device, d, {"voxelResolution": 0.04, "opacityCutoff": 0.1})
    assert np.array_equal(g1.buffer.blockIdx, g2.buffer.blockIdx)
    assert np.array_equal(g1.buffer.maskLo, g2.buffer.maskLo) and np.array_equal(g1.buffer.maskHi, g2.buffer.maskHi)
    assert g1.buffer.count > 100
    o = O.voxelize(d, 0.04, 0.1)
    assert np.array_equal(g2.buffer.blockIdx, o["block_idx"]) and np.array_equal(g2.buffer.maskLo, o["mask_lo"])


def test_user_bounds_and_partial_batches(device):
    d = synth.voxel_1m(30_000)
    g, o = run_both(device, d, res=0.07, cut=0.3, bounds=((-3.1, -2.0, -4.4), (2.3, 5.0, 1.7)))
    assert_same(g, o)


def test_cutoff_extremes(device):
    d = synth.voxel_1m(5_000)
    for cut in (0.0, 0.9995, 1.0, 0.5):
        g, o = run_both(device, d, res=0.2, cut=cut)
        assert_same(g, o)


def test_single_gaussian_closed_form(device):
    d = SplatData(1, np.zeros(3, np.float32), np.array([1, 0, 0, 0], np.float32),
                  np.full(3, math.log(0.1), np.float32), np.array([3.0], np.float32), np.zeros(3, np.float32))
    g = dl.voxelize(device, d, {"voxelResolution": 0.05, "opacityCutoff": 0.1})
    assert g.buffer.popcount() == 504 and g.numBlocksX == 4


def test_reference_order_differs_only_near_cutoff(device):
    d = synth.voxel_1m(60_000)
    g = dl.voxelize(device, d, {"voxelResolution": 0.05, "opacityCutoff": 0.1})
    f = ("block_idx", "mask_lo", "mask_hi", "near_idx", "near_lo", "near_hi")
    ref = O.voxelize(d, 0.05, 0.1, order=1, eps=EPS, fields=f)
    mg = {int(i): (int(l), int(h)) for i, l, h in zip(g.buffer.blockIdx, g.buffer.maskLo, g.buffer.maskHi)}
    mr = {int(i): (int(l), int(h)) for i, l, h in zip(ref["block_idx"], ref["mask_lo"], ref["mask_hi"])}
    near = {int(i): (int(l), int(h)) for i, l, h in zip(ref["near_idx"], ref["near_lo"], ref["near_hi"])}
    differing = 0
    for k in set(mg) | set(mr):
        a, b, n = mg.get(k, (0, 0)), mr.get(k, (0, 0)), near.get(k, (0, 0))
        assert ((a[0] ^ b[0]) & ~n[0]) == 0 and ((a[1] ^ b[1]) & ~n[1]) == 0
        differing += bin(a[0] ^ b[0]).count("1") + bin(a[1] ^ b[1]).count("1")
    print(f"bits differing from the reference order: {differing} (all within eps={EPS})")


@pytest.mark.parametrize("count", [2, 3, 5])
def test_z_row_shards_concatenate_to_the_whole_grid(device, count):
    # each shard voxelizes a contiguous range of z rows of batches; in shard
    # order the block lists concatenate to the unsharded list
    from droplet_b200 import shard
    d = synth.voxel_1m(60_000)
    opts = {"voxelResolution": 0.04, "opacityCutoff": 0.1}
    whole = dl.voxelize(device, d, opts)
    parts = [shard.voxelize_sharded(device, d, opts, i, count) for i in range(count)]
    idx = np.concatenate([p.buffer.blockIdx for p in parts])
    lo = np.concatenate([p.buffer.maskLo for p in parts])
    hi = np.concatenate([p.buffer.maskHi for p in parts])
    assert np.array_equal(idx, whole.buffer.blockIdx)
    assert np.array_equal(lo, whole.buffer.maskLo) and np.array_equal(hi, whole.buffer.maskHi)
    for p in parts:
        assert (p.numBlocksX, p.numBlocksY, p.numBlocksZ) == (whole.numBlocksX, whole.numBlocksY, whole.numBlocksZ)
    assert sum(p.buffer.count > 0 for p in parts) >= 2
    for cut in (0.0,):
        o2 = dict(opts, opacityCutoff=cut)
        w2 = dl.voxelize(device, d, o2)
        p2 = [shard.voxelize_sharded(device, d, o2, i, count) for i in range(count)]
        assert np.array_equal(np.concatenate([p.buffer.blockIdx for p in p2]), w2.buffer.blockIdx)
    with pytest.raises(dl.DropletError):
        dl.voxelize(device, d, dict(opts, shard=(count, count)))


def test_fast_exp_differs_only_near_the_cutoff(device):
    # DL_VOX_FAST_EXP: the hardware ex2 moves a voxel's opacity by ~1e-6 at most;
    # bits may change only where the canonical opacity is within eps of the cutoff
    d = synth.voxel_1m(100_000)
    opts = {"voxelResolution": 0.05, "opacityCutoff": 0.1}
    g = dl.voxelize(device, d, dict(opts, fastExp=True))
    eps = 1e-4
    f = ("block_idx", "mask_lo", "mask_hi", "near_idx", "near_lo", "near_hi", "near_bits")
    o = O.voxelize(d, 0.05, 0.1, eps=eps, fields=f)
    mg = {int(i): (int(l), int(h)) for i, l, h in zip(g.buffer.blockIdx, g.buffer.maskLo, g.buffer.maskHi)}
    mo = {int(i): (int(l), int(h)) for i, l, h in zip(o["block_idx"], o["mask_lo"], o["mask_hi"])}
    near = {int(i): (int(l), int(h)) for i, l, h in zip(o["near_idx"], o["near_lo"], o["near_hi"])}
    differing = 0
    for k in set(mg) | set(mo):
        a, b, n = mg.get(k, (0, 0)), mo.get(k, (0, 0)), near.get(k, (0, 0))
        assert ((a[0] ^ b[0]) & ~n[0]) == 0 and ((a[1] ^ b[1]) & ~n[1]) == 0
        differing += bin(a[0] ^ b[0]).count("1") + bin(a[1] ^ b[1]).count("1")
    print(f"fast exp: {differing} bits differ from the canonical order, all within the {o['near_bits']} bits "
          f"with |alpha - cutoff| < {eps}")
