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


def _query_reference(idx, lo, hi, bmin, res, dims, pts):
    """Occupancy of points by the BlockMaskBuffer rules (block-mask-buffer.ts:41-58,
    duplicates OR-merged as addBlock does) and the voxel grid of voxelize.ts:160-179."""
    table = {}
    for b, l, h in zip(idx.tolist(), lo.tolist(), hi.tolist()):
        ol, oh = table.get(b, (0, 0))
        table[b] = (ol | l, oh | h)
    out = np.zeros(len(pts), np.uint8)
    if not all(math.isfinite(x) for x in list(bmin) + list(dims)) or min(dims) < 1:
        return out
    with np.errstate(invalid="ignore"):
        v = np.floor((pts.astype(np.float64) - np.asarray(bmin, np.float64)) / res)
        inside = np.all((v >= 0) & (v < 4 * np.asarray(dims, np.float64)), axis=1)
    for i in np.nonzero(inside)[0]:
        x, y, z = (int(c) for c in v[i])
        flat = (x >> 2) + (y >> 2) * int(dims[0]) + (z >> 2) * int(dims[0]) * int(dims[1])
        if flat in table:
            bit = (z & 3) * 16 + (y & 3) * 4 + (x & 3)
            l, h = table[flat]
            out[i] = (l >> bit) & 1 if bit < 32 else (h >> (bit - 32)) & 1
    return out


def test_point_queries_match_the_block_mask_buffer(device):
    # dl_vox_query (collision tests against the voxelizer's output) against the
    # BlockMaskBuffer rules on the CPU: random points around the grid, the centres
    # of listed blocks' voxels, non-finite points and the grid's edges
    d = synth.voxel_1m(40_000)
    res = dl.voxelize(device, d, {"voxelResolution": 0.1, "opacityCutoff": 0.1})
    buf = res.buffer
    assert buf.count > 1000
    bmin, bmax = np.asarray(res.bounds.min, np.float64), np.asarray(res.bounds.max, np.float64)
    dims = (res.numBlocksX, res.numBlocksY, res.numBlocksZ)
    rng = np.random.default_rng(5)
    span = bmax - bmin
    p1 = rng.uniform(bmin - 0.1 * span, bmax + 0.1 * span, (60_000, 3))
    pick = rng.integers(0, buf.count, 40_000)
    b = buf.blockIdx[pick].astype(np.int64)
    nx, ny = int(dims[0]), int(dims[1])
    bx, by, bz = b % nx, (b // nx) % ny, b // (nx * ny)
    local = rng.integers(0, 4, (40_000, 3))
    vox = np.stack([bx, by, bz], 1) * 4 + local
    p2 = bmin + (vox + 0.5) * 0.1
    p3 = np.array([[np.nan, 0, 0], [np.inf, 0, 0], [0, -np.inf, 0], list(bmin), list(bmax)], np.float64)
    pts = np.concatenate([p1, p2, p3]).astype(np.float32)
    got = dl.voxelQuery(device, res, pts)
    want = _query_reference(buf.blockIdx, buf.maskLo, buf.maskHi, bmin, 0.1, dims, pts)
    assert np.array_equal(got, want)
    assert 0 < got.sum() < len(pts)
    # a buffer listing blocks twice, their bits split between the copies: OR-merged
    k = min(500, buf.count)
    split = dl.BlockMaskBuffer(np.concatenate([buf.blockIdx, buf.blockIdx[:k]]),
                               np.concatenate([buf.maskLo & np.uint32(0x0000ffff), buf.maskLo[:k]]),
                               np.concatenate([buf.maskHi, np.zeros(k, np.uint32)]))
    merged = dl.BlockMaskBuffer(buf.blockIdx, np.concatenate([buf.maskLo[:k], buf.maskLo[k:] & np.uint32(0x0000ffff)]),
                                buf.maskHi)
    r2 = dl.VoxelizeResult(split, res.bounds, res.voxelResolution, *dims)
    r3 = dl.VoxelizeResult(merged, res.bounds, res.voxelResolution, *dims)
    assert np.array_equal(dl.voxelQuery(device, r2, pts), dl.voxelQuery(device, r3, pts))
    assert np.array_equal(dl.voxelQuery(device, r2, pts),
                          _query_reference(split.blockIdx, split.maskLo, split.maskHi, bmin, 0.1, dims, pts))
    # an empty scene: bounds +-Infinity, nothing solid
    empty = dl.voxelize(device, SplatData.empty(), {"voxelResolution": 0.1})
    assert not dl.voxelQuery(device, empty, pts).any()


def _carve_reference(a, b):
    """A minus B block by block: B's entries OR-merged by index, each of A's entries
    keeps the bits B's do not set, empty entries dropped, A's order kept."""
    table = {}
    for k, l, h in zip(b.blockIdx.tolist(), b.maskLo.tolist(), b.maskHi.tolist()):
        ol, oh = table.get(k, (0, 0))
        table[k] = (ol | l, oh | h)
    out = ([], [], [])
    for k, l, h in zip(a.blockIdx.tolist(), a.maskLo.tolist(), a.maskHi.tolist()):
        bl, bh = table.get(k, (0, 0))
        l, h = l & ~bl & 0xffffffff, h & ~bh & 0xffffffff
        if l or h:
            out[0].append(k)
            out[1].append(l)
            out[2].append(h)
    return [np.asarray(c, np.uint32) for c in out]


@pytest.mark.gpu
def test_carve_matches_the_block_rules(device):
    # dl_vox_carve against the CPU rules: the shell left when a high-cutoff
    # voxelization is carved out of a low-cutoff one, a B with duplicate and
    # absent blocks, and the empty cases
    d = synth.voxel_1m(40_000)
    lo_cut = dl.voxelize(device, d, {"voxelResolution": 0.1, "opacityCutoff": 0.1}).buffer
    hi_cut = dl.voxelize(device, d, {"voxelResolution": 0.1, "opacityCutoff": 0.4}).buffer
    assert lo_cut.count > 1000 and hi_cut.count > 100

    def same(got, want):
        assert np.array_equal(got.blockIdx, want[0])
        assert np.array_equal(got.maskLo, want[1])
        assert np.array_equal(got.maskHi, want[2])

    shell = dl.voxelCarve(device, lo_cut, hi_cut)
    same(shell, _carve_reference(lo_cut, hi_cut))
    assert 0 < shell.count <= lo_cut.count
    rng = np.random.default_rng(11)
    n = lo_cut.count
    pick = rng.integers(0, n, 3 * n // 2)
    absent = np.arange(10**6, 10**6 + 300, dtype=np.uint32)
    b = dl.BlockMaskBuffer(np.concatenate([lo_cut.blockIdx[pick], absent]),
                           rng.integers(0, 2**32, len(pick) + 300, dtype=np.uint64).astype(np.uint32),
                           rng.integers(0, 2**32, len(pick) + 300, dtype=np.uint64).astype(np.uint32))
    same(dl.voxelCarve(device, lo_cut, b), _carve_reference(lo_cut, b))
    empty = dl.BlockMaskBuffer()
    same(dl.voxelCarve(device, lo_cut, empty), (lo_cut.blockIdx, lo_cut.maskLo, lo_cut.maskHi))
    assert dl.voxelCarve(device, lo_cut, lo_cut).count == 0
    assert dl.voxelCarve(device, empty, lo_cut).count == 0
