"""Shared GPU-vs-oracle comparison helpers for the render parity tests."""
import numpy as np

from oracle import oracle as O

ORACLE_FIELDS = ("rgba", "accum", "sorted_idx", "depth_keys", "records", "counts", "tile_list_off",
                 "tile_list_val", "chunk_tile_offsets", "n_visible", "n_pairs")


def bbox_count(bb, max_cov=16384):
    mnx, mny = bb[:, 0] & 0xFFFF, bb[:, 0] >> 16
    mxx, mxy = bb[:, 1] & 0x7FFF, (bb[:, 1] >> 16) & 0x7FFF
    ok = (mxx >= mnx) & (mxy >= mny)
    c = (mxx.astype(np.int64) - mnx + 1) * (mxy.astype(np.int64) - mny + 1)
    return np.where(ok, np.minimum(c, max_cov), 0)


def gpu_render_debug(renderer, data, cam, bg=None):
    renderer.set_debug(True)
    rgba = renderer.render(data, cam, bg)
    g = {"rgba": rgba,
         "nvis": int(renderer.debug_get("nvis", np.uint64)[0]),
         "npairs": int(renderer.debug_get("npairs", np.uint64)[0]),
         "depth_keys": renderer.debug_get("depth_keys", np.uint32),
         "sorted_idx": renderer.debug_get("sorted_idx", np.uint32),
         "recA": renderer.debug_get("recA", np.float32).reshape(-1, 4),
         "recBC": renderer.debug_get("recBC", np.float32).reshape(-1, 8),
         "bbox": renderer.debug_get("bbox", np.uint32).reshape(-1, 2),
         "tile_off": renderer.debug_get("tile_off", np.uint32),
         "pair_vals": renderer.debug_get("pair_vals", np.uint32),
         "accum": renderer.debug_get("accum", np.float32)}
    return g


def assert_render_parity(g, o, max_cov=16384):
    """Bit-exact comparison of every stage of one view (single-chunk oracle)."""
    nv = o["n_visible"]
    assert g["nvis"] == nv
    assert np.array_equal(g["sorted_idx"][:nv], o["sorted_idx"]), "depth order differs"
    assert np.array_equal(g["depth_keys"][:nv], o["depth_keys"]), "depth keys differ"
    idx = o["sorted_idx"].astype(np.int64)
    rec = o["records"].reshape(-1, 12)
    gA = g["recA"][idx]
    assert np.array_equal(gA.view(np.uint32), rec[:, 0:4].view(np.uint32)), "projected slot 0 differs"
    live = rec[:, 2] > 0
    gBC = g["recBC"][idx]
    assert np.array_equal(gBC[live][:, 0:4].view(np.uint32), rec[live][:, 4:8].view(np.uint32)), "conic/alpha differ"
    assert np.array_equal(gBC[live][:, 4:7].view(np.uint32), rec[live][:, 8:11].view(np.uint32)), "colour differs"
    assert np.array_equal(bbox_count(g["bbox"][idx], max_cov), o["counts"].astype(np.int64)), "tile counts differ"
    assert g["npairs"] == o["n_pairs"]
    assert np.array_equal(g["tile_off"], o["chunk_tile_offsets"] if o["n_pairs"] else np.zeros_like(g["tile_off"]))
    rank = np.empty(max(int(idx.max()) + 1 if nv else 1, 1), np.int64)
    rank[idx] = np.arange(nv)
    pv = g["pair_vals"].astype(np.int64)
    phantom = ((pv >> 31) & 1).astype(bool)
    splat = pv & 0x3FFFFFFF
    assert np.array_equal(rank[splat], o["tile_list_val"].astype(np.int64)), "tile pair lists differ"
    # the flag marks exactly the splats whose box lies wholly left of / above the image
    rA = g["recA"][splat]
    wholly_out = (np.floor((rA[:, 0] + rA[:, 2]) / 16) < 0) | (np.floor((rA[:, 1] + rA[:, 2]) / 16) < 0)
    assert np.array_equal(phantom, wholly_out), "phantom flags differ"
    assert np.array_equal(g["rgba"], o["rgba"]), "RGBA8 differs"
    assert np.array_equal(g["accum"].view(np.uint32), o["accum"].view(np.uint32)), "f32 accumulator differs"
