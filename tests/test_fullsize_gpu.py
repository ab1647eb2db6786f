"""Full-size parity of the configurations the benchmark measures.

* ring64 — the headline batch exactly as bench.py times it: the 3M-Gaussian
  SH3 scene uploaded with FP16 SH, flags F16_RECORDS | FAST_EXP |
  CULL_OFFSCREEN, autotuned knobs, the trained tile-cost model attached,
  images written to device memory.  One view of each ring resolution is
  compared with the f32 oracle (RGBA8 within +-1 LSB on >= 99.9% of pixels)
  and with the FP64 oracle (max / mean error reported); the exact f32 path
  must match the f32 oracle bit for bit on the same views; the public
  host-in / host-out call (the e2e number) must give the batch's pixels for
  all 64 views.
* voxel1m — config 2 at full size (1M Gaussians, res 0.05): bit-exact against
  the canonical-order oracle; against the reference-order oracle (its BVH
  summation order) bits differ only where |alpha - cutoff| < eps, counted.
* zipf10m — config 5's grid (10M Zipf Gaussians, res 0.02): the GPU grid is
  compared z row of 16^3-block batches by z row against the oracle run on
  the same rows (an edge row, the densest row, and one between), and the
  sharded call concatenates to the whole grid.

Run with -s to see the error and epsilon-band tables.
"""
import numpy as np
import pytest

import droplet_b200 as dl
from droplet_b200 import _lib, learned, shard, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

EPS = 1e-5
HEADLINE = _lib.DL_BATCH_F16_RECORDS | _lib.DL_BATCH_FAST_EXP | _lib.DL_BATCH_CULL_OFFSCREEN


def _f64_bytes(acc64):
    """Composite over the default background (0, 0, 0, 1) in f64: bytes before rounding."""
    a = acc64.reshape(-1, 4)
    rgb = np.clip(a[:, :3], 0.0, 1.0) * 255.0
    alpha = np.clip(1.0 - a[:, 3] + a[:, 3] * 1.0, 0.0, 1.0) * 255.0
    return np.concatenate([rgb, alpha[:, None]], axis=1)


@pytest.fixture(scope="module")
def sh3_scene():
    return synth.sh3_3m()


def test_ring64_headline_batch_against_oracle(device, sh3_scene):
    import torch
    data = sh3_scene
    cams = synth.ring_cameras(64)
    r = dl.Renderer(device)
    stream = torch.cuda.Stream()
    r.set_stream(stream.cuda_stream)
    scene = r.upload(data, "f16")
    tuning = r.autotune(scene, cams, flags=HEADLINE, reps=1)
    model = learned.load_default(device)
    assert model is not None, "the committed tile-cost model must load"
    r.set_scheduler(model)
    outs = [torch.empty(c.width * c.height * 4, dtype=torch.uint8, device="cuda") for c in cams]
    r.render_batch(scene, cams, flags=HEADLINE, outs=[o.data_ptr() for o in outs])
    torch.cuda.synchronize()
    batch = [o.cpu().numpy() for o in outs]

    # the public host-in / host-out call renders the same pixels for every view
    r2 = dl.Renderer(device)
    many = r2.render_many(data, cams, flags=HEADLINE | _lib.DL_BATCH_SH16)
    for k in range(64):
        assert np.array_equal(many[k], batch[k]), f"render_many differs from the batch in view {k}"
    r2.destroy()

    # exact f32 path on the compared views
    check = [0, 1, 2, 3]                   # 640x360, 1280x720, 1920x1080, 2560x1440
    scene32 = r.upload(data, "f32")
    exact = r.render_batch(scene32, [cams[k] for k in check], flags=0)
    scene32.destroy()
    lines = [f"ring64 headline batch, tuning {tuning}"]
    for j, k in enumerate(check):
        cam = cams[k]
        o = O.render(data, cam, f64=True, fields=("rgba", "accum64"))
        ref32 = o["rgba"].reshape(-1, 4).astype(np.int16)
        got = batch[k].reshape(-1, 4)
        diff = np.abs(got.astype(np.int16) - ref32).max(axis=1)
        within = float((diff <= 1).mean())
        e64 = np.abs(got.astype(np.float64) - _f64_bytes(o["accum64"]))
        x64 = np.abs(exact[j].reshape(-1, 4).astype(np.float64) - _f64_bytes(o["accum64"]))
        lines.append(f"  view {k:2d} {cam.width}x{cam.height}: within 1 LSB of f32 oracle {within * 100:.4f}% "
                     f"(max diff {int(diff.max())}); vs f64: max {e64.max():.3f} LSB mean {e64.mean():.4f} LSB; "
                     f"exact f32 path vs f64: max {x64.max():.3f} mean {x64.mean():.4f}")
        assert within >= 0.999, (k, within)
        assert np.array_equal(exact[j], o["rgba"]), f"exact path differs from the f32 oracle in view {k}"
    scene.destroy()
    r.destroy()
    print("\n" + "\n".join(lines))


def _eps_band_count(gpu_idx, gpu_lo, gpu_hi, ref):
    """Bits where the GPU grid and the reference-order grid differ; every one
    must lie in the reference's |alpha - cutoff| < eps band."""
    mg = {int(i): (int(l), int(h)) for i, l, h in zip(gpu_idx, gpu_lo, gpu_hi)}
    mr = {int(i): (int(l), int(h)) for i, l, h in zip(ref["block_idx"], ref["mask_lo"], ref["mask_hi"])}
    near = {int(i): (int(l), int(h)) for i, l, h in zip(ref["near_idx"], ref["near_lo"], ref["near_hi"])}
    differing = 0
    for k in set(mg) | set(mr):
        a, b, n = mg.get(k, (0, 0)), mr.get(k, (0, 0)), near.get(k, (0, 0))
        assert ((a[0] ^ b[0]) & ~n[0]) == 0 and ((a[1] ^ b[1]) & ~n[1]) == 0, f"bit outside the eps band, block {k}"
        differing += bin(a[0] ^ b[0]).count("1") + bin(a[1] ^ b[1]).count("1")
    return differing


REF_FIELDS = ("block_idx", "mask_lo", "mask_hi", "near_idx", "near_lo", "near_hi", "near_bits")


def test_voxel1m_full_size(device):
    d = synth.voxel_1m()
    opts = {"voxelResolution": 0.05, "opacityCutoff": 0.1}
    g = dl.voxelize(device, d, opts)
    o = O.voxelize(d, 0.05, 0.1)
    assert np.array_equal(g.buffer.blockIdx, o["block_idx"]), "block list / order differs"
    assert np.array_equal(g.buffer.maskLo, o["mask_lo"]) and np.array_equal(g.buffer.maskHi, o["mask_hi"])
    assert np.array_equal([g.numBlocksX, g.numBlocksY, g.numBlocksZ], o["dims"])
    ref = O.voxelize(d, 0.05, 0.1, order=1, eps=EPS, fields=REF_FIELDS)
    diff = _eps_band_count(g.buffer.blockIdx, g.buffer.maskLo, g.buffer.maskHi, ref)
    # the hardware-exp variant against the canonical order, band 1e-4
    fast = dl.voxelize(device, d, dict(opts, fastExp=True))
    canon = O.voxelize(d, 0.05, 0.1, eps=1e-4, fields=REF_FIELDS)
    fdiff = _eps_band_count(fast.buffer.blockIdx, fast.buffer.maskLo, fast.buffer.maskHi, canon)
    print(f"\nvoxel1m: {g.buffer.count} blocks, {g.buffer.popcount()} solid voxels; bit-exact vs canonical order; "
          f"vs reference order {diff} bits differ, all within the {ref['near_bits']} bits with "
          f"|alpha - cutoff| < {EPS}; hardware-exp variant: {fdiff} bits differ from the canonical order, all "
          f"within the {canon['near_bits']} bits with |alpha - cutoff| < 1e-4")


def test_zipf10m_grid_by_z_rows(device):
    d = synth.zipf_10m()
    res = 0.02
    opts = {"voxelResolution": res, "opacityCutoff": 0.1}
    g = dl.voxelize(device, d, opts)
    nx, ny, nz = int(g.numBlocksX), int(g.numBlocksY), int(g.numBlocksZ)
    zrow = (g.buffer.blockIdx.astype(np.int64) // (nx * ny)) // 16
    rows_total = (nz + 15) // 16
    # blocks per z row: the densest row carries the most
    counts = np.bincount(zrow, minlength=rows_total)
    dense = int(np.argmax(counts))
    rows = sorted({0, dense, min(rows_total - 1, (dense + rows_total) // 2)})
    lines = [f"zipf10m: grid {nx}x{ny}x{nz} blocks ({rows_total} z rows of batches), {g.buffer.count} blocks"]
    for zr in rows:
        sel = zrow == zr
        o = O.voxelize(d, res, 0.1, z_rows=(zr, zr + 1), fields=("block_idx", "mask_lo", "mask_hi", "dims"))
        assert np.array_equal(o["dims"], [nx, ny, nz])
        assert np.array_equal(g.buffer.blockIdx[sel], o["block_idx"]), f"z row {zr}: block list differs"
        assert np.array_equal(g.buffer.maskLo[sel], o["mask_lo"]) and np.array_equal(g.buffer.maskHi[sel],
                                                                                      o["mask_hi"])
        line = f"  z row {zr:2d}: {int(sel.sum())} blocks bit-exact vs canonical order"
        if zr == dense:
            ref = O.voxelize(d, res, 0.1, order=1, eps=EPS, fields=REF_FIELDS, z_rows=(zr, zr + 1))
            diff = _eps_band_count(g.buffer.blockIdx[sel], g.buffer.maskLo[sel], g.buffer.maskHi[sel], ref)
            line += (f"; vs reference order {diff} bits differ, all within the {ref['near_bits']} bits with "
                     f"|alpha - cutoff| < {EPS}")
        lines.append(line)
    # the sharded call (z-row ranges balanced by pair counts) concatenates to the grid
    parts = [shard.voxelize_sharded(device, d, opts, i, 4) for i in range(4)]
    assert np.array_equal(np.concatenate([p.buffer.blockIdx for p in parts]), g.buffer.blockIdx)
    assert np.array_equal(np.concatenate([p.buffer.maskLo for p in parts]), g.buffer.maskLo)
    assert np.array_equal(np.concatenate([p.buffer.maskHi for p in parts]), g.buffer.maskHi)
    lines.append("  4 z-row shards concatenate to the whole grid")
    print("\n" + "\n".join(lines))
