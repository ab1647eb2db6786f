"""GPU parity of the renderer against the oracle, through the C ABI.

Integer stages (depth keys, depth order, tile counts, tile offsets, per-tile
pair lists) must be bit-exact, and so must the projected records, the f32
accumulator and the RGBA8 bytes: the kernels evaluate the shaders' f32
expressions in the same order with FMA contraction off and share dl_math.h's
exp/atan2/asin with the oracle.  Variants that trade exactness for speed (f16
records, hardware exp) are held to the stated tolerance: RGBA8 within +-1 LSB
on >= 99.9% of pixels."""
import math

import numpy as np
import pytest

import droplet_b200 as dl
from droplet_b200 import _lib, synth
from droplet_b200.types import RenderCamera, SplatData, mat4LookAt
from oracle import oracle as O
from parity import ORACLE_FIELDS, assert_render_parity, gpu_render_debug

pytestmark = pytest.mark.gpu


def nonblack(rgba):
    p = rgba.reshape(-1, 4)
    return int(((p[:, 0] > 5) | (p[:, 1] > 5) | (p[:, 2] > 5)).sum())


def check(renderer, data, cam, bg=(0.0, 0.0, 0.0, 1.0), max_cov=16384):
    g = gpu_render_debug(renderer, data, cam, bg)
    o = O.render(data, cam, bg, maxCoverage=max_cov, chunkCap=1 << 30, fields=ORACLE_FIELDS)
    assert_render_parity(g, o, max_cov)
    return g, o


# ---- the reference's browser tests (examples/browser/test.ts), on the GPU path
def test_empty_scene(renderer):
    rgba = renderer.render(SplatData.empty(), synth.front_camera())
    assert nonblack(rgba) == 0 and rgba.reshape(-1, 4)[0, 3] == 255


def test_one_splat(renderer):
    g, o = check(renderer, synth.one_splat((0, 0, 0)), synth.front_camera())
    img = g["rgba"].reshape(128, 128, 4)[..., 0]
    assert img[64, 64] > 100 and abs(int(img[64, 54]) - int(img[64, 74])) < 10


def test_three_splats_and_occlusion(renderer):
    d = SplatData(3, [0, 0, 1, 0.5, 0, 0.8, -0.5, 0.3, 0.8], [1, 0, 0, 0] * 3, [-2.5] * 9, [3, 3, 3],
                  [0.5, -0.5, -0.5, -0.5, 0.5, -0.5, -0.5, -0.5, 0.5])
    check(renderer, d, synth.front_camera(256, 256))
    d2 = SplatData(2, [0, 0, 1, 0, 0, -1], [1, 0, 0, 0] * 2, [-2.5] * 6, [4, 4], [0.5, -0.5, -0.5, -0.5, 0.5, -0.5])
    g, _ = check(renderer, d2, synth.front_camera())
    px = g["rgba"].reshape(128, 128, 4)[64, 64]
    assert px[0] > 200 and px[1] < 50


def test_sphere_disc(renderer):
    g, _ = check(renderer, synth.many_splats(5000, "sphere"), synth.front_camera(256, 256))
    assert 10000 < nonblack(g["rgba"]) < 30000


def test_chunk_cap_has_no_effect(device):
    d = synth.many_splats(200_000, "random")
    a = dl.Renderer(device).render(d, synth.front_camera(64, 64))
    b = dl.Renderer(device, {"chunkCap": 50_000}).render(d, synth.front_camera(64, 64))
    o = O.render(d, synth.front_camera(64, 64), chunkCap=50_000)
    assert np.array_equal(a, b) and np.array_equal(a, o["rgba"])


def test_dense_large_splats(renderer):
    n = 200_000
    rng = np.random.default_rng(7)
    pos = ((rng.random((n, 3)) - 0.5) * 0.1).astype(np.float32)
    rot = np.zeros((n, 4), np.float32); rot[:, 0] = 1
    dc = np.zeros((n, 3), np.float32); dc[:, 0] = 0.5
    d = SplatData(n, pos, rot, np.full((n, 3), -2.5, np.float32), np.zeros(n, np.float32), dc)
    g, _ = check(renderer, d, synth.front_camera(256, 256))
    assert nonblack(g["rgba"]) > 100


def test_one_million_random(renderer):
    g, _ = check(renderer, synth.many_splats(1_000_000, "random"), synth.front_camera(256, 256))
    assert nonblack(g["rgba"]) > 1000


# ---- seeded workloads
def test_plain_100k_720p_full_size(renderer):
    check(renderer, synth.plain_100k(), synth.plain_100k_camera(), bg=(0.1, 0.2, 0.3, 0.5))


@pytest.mark.parametrize("bands", [1, 2, 3])
def test_sh_bands_1080p(renderer, bands):
    d = synth.cluster_scene(150_000, seed=20 + bands, clusters=32, extent=10.0, bands=bands)
    check(renderer, d, synth.pinhole(1920, 1080, (0.0, 2.0, 12.0)))


def test_equirect(renderer):
    d = synth.cluster_scene(150_000, seed=31, clusters=32, extent=10.0, bands=3)
    check(renderer, d, synth.sh3_3m_cameras()[1])


def test_max_coverage_truncation(device):
    r = dl.Renderer(device, {"maxCoveragePerSplat": 7})
    d = synth.cluster_scene(20_000, seed=4, clusters=4, extent=1.0, log_lo=0.05, log_hi=0.3)
    check(r, d, synth.pinhole(640, 360, (0.0, 0.0, 3.0)), max_cov=7)


def test_offscreen_left_top_splats_bin_to_edge_tiles(renderer):
    # u32() saturation in project.ts:224-227: off-screen splats to the left/top
    # still count tiles in column/row 0; the pair lists must reproduce that.
    rng = np.random.default_rng(3)
    n = 5000
    pos = np.c_[rng.uniform(-30, 30, n), rng.uniform(-30, 30, n), rng.uniform(-5, 1, n)].astype(np.float32)
    rot = np.zeros((n, 4), np.float32); rot[:, 0] = 1
    d = SplatData(n, pos, rot, np.full((n, 3), -2.0, np.float32), np.ones(n, np.float32),
                  rng.normal(0, .5, (n, 3)).astype(np.float32))
    g, o = check(renderer, d, synth.pinhole(320, 240, (0.0, 0.0, 4.0)))
    assert o["n_pairs"] > 0


def test_near_far_and_degenerate(renderer):
    rng = np.random.default_rng(9)
    n = 4000
    pos = np.c_[rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), rng.uniform(3.0, 5.0, n)].astype(np.float32)
    q = rng.normal(0, 1, (n, 4)); q /= np.linalg.norm(q, axis=1, keepdims=True)
    ls = rng.uniform(-12, 1, (n, 3)).astype(np.float32)          # needles, sub-pixel and screen-filling
    d = SplatData(n, pos, q.astype(np.float32), ls, rng.normal(0, 3, n).astype(np.float32),
                  rng.normal(0, .5, (n, 3)).astype(np.float32))
    cam = RenderCamera(300, 200, mat4LookAt((0, 0, 4), (0, 0, 0), (0, 1, 0)), math.pi / 3, 0.5, 3.9)
    check(renderer, d, cam)


def test_odd_sizes(renderer):
    d = synth.plain_100k(30_000)
    for w, h in ((1, 1), (17, 33), (255, 1), (1000, 7)):
        check(renderer, d, synth.pinhole(w, h, (0.0, 0.0, 4.0)))


# ---- batched path: same pixels as the single-view path
def test_batch_matches_single_views(device, renderer):
    d = synth.cluster_scene(200_000, seed=12, clusters=64, extent=10.0, bands=3)
    cams = synth.ring_cameras(6, resolutions=[(320, 180), (640, 360), (500, 400)])
    single = [renderer.render(d, c) for c in cams]
    r2 = dl.Renderer(device)
    sc = r2.upload(d)
    plain = r2.render_batch(sc, cams, flags=_lib.DL_BATCH_PLAIN)
    batched = r2.render_batch(sc, cams)
    for a, b, c in zip(single, plain, batched):
        assert np.array_equal(a, b) and np.array_equal(a, c)


def test_view_shards_reassemble_the_batch(device, renderer):
    # each rank of a world renders its round-robin share; together they equal
    # the single-GPU batch (ranks emulated one after another on this GPU)
    from droplet_b200 import shard
    d = synth.cluster_scene(80_000, seed=15, clusters=16, extent=10.0, bands=2)
    cams = synth.ring_cameras(7, resolutions=[(320, 180), (256, 256)])
    r2 = dl.Renderer(device)
    sc = r2.upload(d)
    whole = r2.render_batch(sc, cams)
    got = [None] * len(cams)
    for rank in range(3):
        ids, imgs = shard.render_views_sharded(r2, sc, cams, rank, 3)
        for i, im in zip(ids, imgs):
            got[i] = im
    for a, b in zip(whole, got):
        assert np.array_equal(a, b)


def test_graph_replay_follows_new_cameras(device, renderer):
    # the batched frame is captured once and replayed; camera tables are
    # uploaded before every replay, so a moved ring must still match
    d = synth.cluster_scene(100_000, seed=14, clusters=32, extent=10.0, bands=1)
    r2 = dl.Renderer(device)
    sc = r2.upload(d)
    for radius in (12.0, 9.0, 15.0):
        cams = synth.ring_cameras(5, radius=radius, resolutions=[(320, 180), (400, 300)])
        got = r2.render_batch(sc, cams)
        nog = r2.render_batch(sc, cams, flags=_lib.DL_BATCH_NO_GRAPH)
        for g, n, c in zip(got, nog, cams):
            assert np.array_equal(g, n) and np.array_equal(g, renderer.render(d, c))


def _lsb_share(a, b):
    diff = np.abs(a.astype(np.int16) - b.astype(np.int16)).reshape(-1, 4).max(axis=1)
    return float((diff <= 1).mean()), int(diff.max())


@pytest.mark.parametrize("flags,prec", [(_lib.DL_BATCH_F16_RECORDS, "f32"), (_lib.DL_BATCH_F16_RECORDS, "f16"),
                                        (_lib.DL_BATCH_F16_RECORDS, "bf16"), (_lib.DL_BATCH_FAST_EXP, "f32")])
def test_precision_variants_within_one_lsb(device, flags, prec):
    d = synth.cluster_scene(200_000, seed=13, clusters=64, extent=10.0, bands=3)
    cam = synth.pinhole(960, 540, (0.0, 2.0, 12.0))
    o = O.render(d, cam)["rgba"]
    r = dl.Renderer(device)
    sc = r.upload(d, prec)
    got = r.render_batch(sc, [cam], flags=flags)[0]
    share, worst = _lsb_share(got, o)
    assert share >= 0.999, (share, worst)


def test_tuning_knobs_change_no_pixel_and_autotune_keeps_one(device):
    # every knob of dl_tuning changes timing only: the images must be identical
    d = synth.cluster_scene(150_000, seed=16, clusters=32, extent=10.0, bands=3)
    cams = synth.ring_cameras(6, resolutions=[(640, 360), (333, 257), (1280, 720)])
    r2 = dl.Renderer(device)
    sc = r2.upload(d, "f16")
    flags = _lib.DL_BATCH_F16_RECORDS | _lib.DL_BATCH_FAST_EXP
    base = r2.render_batch(sc, cams, flags=flags)
    for kw in ({"pair_sort_bits": 7}, {"pair_sort_bits": 6}, {"raster_shape": "16x2"}, {"raster_shape": "4x8"},
               {"raster_shape": "8x8x2"}, {"raster_shape": "8x4-f32x2"}, {"raster_shape": "tile-f32x2"},
               {"raster_shape": "tile-f32x2", "bin_tile": "32x8"}, {"raster_shape": "tile-f32x2", "bin_tile": "8x8"},
               {"raster_shape": "tile"}, {"raster_shape": "tile", "bin_tile": "32x8"},
               {"raster_shape": "tile", "bin_tile": "8x8"},
               {"raster_ctas_per_sm": 3}, {"raster_ctas_per_sm": 1},
               {"pair_sort_bits": 6, "raster_shape": "4x8", "raster_ctas_per_sm": 2},
               {"bin_tile": "8x8"}, {"bin_tile": "32x8"}, {"bin_tile": "8x8", "raster_shape": "8x8x2"},
               {"bin_tile": "8x8", "raster_shape": "16x2"}, {"bin_tile": "32x8", "raster_shape": "8x4-f32x2"},
               {"bin_tile": "32x8", "raster_shape": "4x8", "pair_sort_bits": 6}):
        r2.set_tuning(**kw)
        for a, b in zip(base, r2.render_batch(sc, cams, flags=flags)):
            assert np.array_equal(a, b), kw
    r2.set_tuning(raster_shape="8x8x2")
    sc32 = r2.upload(d)
    for a, c in zip(r2.render_batch(sc32, cams), cams):     # exact path, two pixels per lane
        assert np.array_equal(a, renderer_single(device, d, c))
    r2.set_tuning(pair_sort_bits=6, raster_shape="4x8", raster_ctas_per_sm=2)
                                           # exact path under the last tuning == the single-view render
    exact = r2.render_batch(sc32, cams)
    for a, c in zip(exact, cams):
        assert np.array_equal(a, renderer_single(device, d, c))
    for tile in ("8x8", "32x8"):           # exact path binned with other tiles, bit-exact too
        r2.set_tuning(bin_tile=tile)
        for a, c in zip(r2.render_batch(sc32, cams), cams):
            assert np.array_equal(a, renderer_single(device, d, c)), tile
    for tile in ("16x16", "32x8"):         # exact path, one CTA per tile
        r2.set_tuning(raster_shape="tile", bin_tile=tile)
        for a, c in zip(r2.render_batch(sc32, cams), cams):
            assert np.array_equal(a, renderer_single(device, d, c)), tile
    r2.set_tuning()
    t = r2.autotune(sc, cams, flags=flags, reps=2)
    assert t["pair_sort_bits"] in (6, 7, 8) and t["raster_shape"] in dl.Renderer.RASTER_SHAPES and t["frame_ms"] > 0
    assert t["bin_tile"] in dl.Renderer.BIN_TILES
    assert r2.get_tuning() == {k: t[k] for k in ("pair_sort_bits", "raster_shape", "raster_ctas_per_sm", "bin_tile")}
    for a, b in zip(base, r2.render_batch(sc, cams, flags=flags)):
        assert np.array_equal(a, b)
    with pytest.raises(dl.DropletError):
        r2.set_tuning(pair_sort_bits=9)


def renderer_single(device, d, cam):
    r = dl.Renderer(device)
    try:
        return r.render(d, cam)
    finally:
        r.destroy()


def test_other_binning_tiles_keep_the_coverage_truncation(device):
    # with a maxCoveragePerSplat below the view's 16x16 tile count a large splat
    # keeps only a row-major prefix of its 16x16 tiles; a tuned binning tile must
    # not change that, so such frames bin with 16x16 tiles
    n = 400
    rng = np.random.default_rng(9)
    d = dl.SplatData(n, (rng.random((n, 3)) * 0.4 - 0.2).astype(np.float32),
                     np.tile(np.array([1, 0, 0, 0], np.float32), (n, 1)), np.full((n, 3), np.log(0.4), np.float32),
                     rng.normal(0.0, 1.0, n).astype(np.float32), rng.normal(0.0, 0.5, (n, 3)).astype(np.float32))
    cam = synth.pinhole(320, 240, (0.0, 0.0, 3.0))
    want = O.render(d, cam, maxCoverage=40)["rgba"]
    for tile in ("8x8", "32x8"):
        r = dl.Renderer(device, {"maxCoveragePerSplat": 40})
        r.set_tuning(bin_tile=tile)
        sc = r.upload(d)
        assert np.array_equal(r.render_batch(sc, [cam, cam])[1], want), tile
        assert np.array_equal(r.render(d, cam), want), tile
        sc.destroy()
        r.destroy()


def test_render_many_groups_and_sh16_match_the_batch(device):
    # host outputs of 8+ views: the scene uploads in eight splat ranges, each
    # projected when it has arrived, and the rasterizer runs per view range with
    # overlapped read-back; DL_BATCH_SH16 keeps the uploaded SH in f16 like a
    # Scene uploaded as "f16".  The splat count is not a multiple of 4.
    d = synth.cluster_scene(120_003, seed=17, clusters=24, extent=10.0, bands=3)
    cams = synth.ring_cameras(10, resolutions=[(320, 180), (200, 120), (640, 360)])
    r2 = dl.Renderer(device)
    sc32, sc16 = r2.upload(d), r2.upload(d, "f16")
    # references: batches of fewer than 8 views take the ungrouped path
    ref32 = r2.render_batch(sc32, cams[:5]) + r2.render_batch(sc32, cams[5:])
    got32 = r2.render_many(d, cams)
    for a, b in zip(ref32, got32):
        assert np.array_equal(a, b)
    fl = _lib.DL_BATCH_F16_RECORDS | _lib.DL_BATCH_FAST_EXP
    ref16 = r2.render_batch(sc16, cams[:5], flags=fl) + r2.render_batch(sc16, cams[5:], flags=fl)
    got16 = r2.render_many(d, cams, flags=fl | _lib.DL_BATCH_SH16)
    for a, b in zip(ref16, got16):
        assert np.array_equal(a, b)
    fl |= _lib.DL_BATCH_CULL_OFFSCREEN
    got = r2.render_batch(sc16, cams, flags=fl)
    for a, b in zip(ref16, got):
        assert np.array_equal(a, b)
    got = r2.render_many(d, cams, flags=fl | _lib.DL_BATCH_SH16)
    for a, b in zip(ref16, got):
        assert np.array_equal(a, b)
    # fewer splats than upload ranges: empty ranges are skipped
    tiny = synth.cluster_scene(5, seed=18, clusters=2, extent=1.0, bands=3)
    cams8 = synth.ring_cameras(8, radius=4.0, resolutions=[(160, 96)])
    st = r2.upload(tiny, "f16")
    ref = r2.render_batch(st, cams8[:4], flags=fl) + r2.render_batch(st, cams8[4:], flags=fl)
    got = r2.render_many(tiny, cams8, flags=fl | _lib.DL_BATCH_SH16)
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)
    assert any(np.asarray(a).reshape(-1, 4)[:, 3].any() for a in ref)


@pytest.mark.parametrize("op_mu", [0.0, -3.0])
def test_offscreen_cull_changes_no_pixel(device, renderer, op_mu):
    # splats whose tile box misses the image (or only has phantom tiles), or
    # whose opacity keeps alpha below 1/255 everywhere, leave the depth order;
    # the others are binned by the box of the ellipse outside which their alpha
    # is below 1/255 (smaller for lower opacity).  Every tile list keeps its
    # order, so pixels are unchanged.  op_mu -3: most opacities below 0.1.
    d = synth.cluster_scene(150_000, seed=19, clusters=32, extent=10.0, bands=2, op_mu=op_mu)
    cams = synth.ring_cameras(5, resolutions=[(320, 180), (500, 280)]) + [synth.pinhole(256, 256, (0.0, 0.0, 0.5))]
    r2 = dl.Renderer(device)
    sc = r2.upload(d)
    for flags in (0, _lib.DL_BATCH_F16_RECORDS | _lib.DL_BATCH_FAST_EXP):
        a = r2.render_batch(sc, cams, flags=flags)
        b = r2.render_batch(sc, cams, flags=flags | _lib.DL_BATCH_CULL_OFFSCREEN)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    # the cull mode's screen record (box half-extents) through the other fast rasterizers
    fast = _lib.DL_BATCH_F16_RECORDS | _lib.DL_BATCH_FAST_EXP
    a = r2.render_batch(sc, cams, flags=fast)
    for shape in ("tile", "8x4-f32x2", "8x4"):
        r2.set_tuning(raster_shape=shape)
        for x, y in zip(a, r2.render_batch(sc, cams, flags=fast | _lib.DL_BATCH_CULL_OFFSCREEN)):
            assert np.array_equal(x, y), shape
    r2.set_tuning()
    one = r2.render_batch(sc, cams[:1], flags=_lib.DL_BATCH_CULL_OFFSCREEN)[0]
    assert np.array_equal(one, renderer.render(d, cams[0]))
    assert int(r2.debug_get("nvis", np.uint64)[0]) < d.count


def test_cull_mode_near_the_image_edges(device, renderer):
    # The cull mode drops splat-views whose tile box misses the image.  Splats
    # straddling the frustum's edges, strongly anisotropic, with unnormalised
    # rotations: the pixels are those of the frame without the cull mode and,
    # in the exact arithmetic, of the oracle.
    rng = np.random.default_rng(23)
    n = 40_000
    cam = synth.pinhole(640, 360, (0.0, 0.0, 4.0))
    half_h = math.tan(math.pi / 6)
    half_w = half_h * 640 / 360
    z = rng.uniform(0.5, 8.0, n)                    # distance in front of the camera
    side = rng.integers(0, 4, n)
    u = rng.uniform(-1.3, 1.3, n)
    edge = rng.uniform(0.9, 1.4, n)                 # in units of the half-width: inside and outside
    x = np.where(side < 2, np.where(side == 0, -1, 1) * edge * half_w, u * half_w) * z
    y = np.where(side >= 2, np.where(side == 2, -1, 1) * edge * half_h, u * half_h) * z
    pos = np.stack([x, y, 4.0 - z], 1)
    q = rng.normal(0.0, 1.0, (n, 4)) * rng.uniform(0.5, 2.0, (n, 1))
    ls = np.stack([rng.uniform(math.log(0.05), math.log(0.6), n), rng.uniform(math.log(0.002), math.log(0.02), n),
                   rng.uniform(math.log(0.002), math.log(0.05), n)], 1)
    d = SplatData(n, pos.astype(np.float32), q.astype(np.float32), ls.astype(np.float32),
                  rng.normal(1.0, 1.5, n).astype(np.float32), rng.normal(0.0, 0.5, (n, 3)).astype(np.float32))
    r2 = dl.Renderer(device)
    sc = r2.upload(d)
    cams = [cam, synth.pinhole(333, 257, (0.5, -0.3, 3.0))]
    fast = _lib.DL_BATCH_F16_RECORDS | _lib.DL_BATCH_FAST_EXP
    for flags in (0, fast):
        a = r2.render_batch(sc, cams, flags=flags)
        b = r2.render_batch(sc, cams, flags=flags | _lib.DL_BATCH_CULL_OFFSCREEN)
        for x0, y0 in zip(a, b):
            assert np.array_equal(x0, y0), flags
    exact = r2.render_batch(sc, cams, flags=_lib.DL_BATCH_CULL_OFFSCREEN)
    for img, c in zip(exact, cams):
        assert np.array_equal(img, O.render(d, c)["rgba"])


def test_ply_parsed_into_pinned_memory_renders_like_its_data(renderer, tmp_path):
    # dl_ply_load parses the file into page-locked arrays; rendering them is
    # bit-exact with the same splats loaded by the Python loader, and with the oracle
    from droplet_b200 import ply
    d = synth.cluster_scene(20_000, seed=8, clusters=8, extent=1.5, bands=3)
    path = str(tmp_path / "scene.ply")
    ply.savePlySplats(d, path)
    p = dl.PlySplats(path, pinned=True)
    cam = synth.pinhole(640, 360, (0.0, 0.3, 4.0))
    got = renderer.render(p.data, cam)
    assert np.array_equal(got, renderer.render(ply.loadPlySplats(path), cam))
    assert np.array_equal(got, O.render(p.data, cam)["rgba"])
    sc = renderer.upload(p.data, "f32")
    assert np.array_equal(renderer.render_batch(sc, [cam])[0], got)
    sc.destroy()
    p.destroy()
