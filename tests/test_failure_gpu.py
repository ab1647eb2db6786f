"""Failure paths, made on purpose without faulting the GPU.

* Bounded waits: every decoupled look-back polls an unpublished predecessor
  at most a settable number of times.  A test hook makes one CTA of a stage
  withhold its status (a flag that nothing else sets), so its successors run
  into a short limit; the call must come back with DL_E_TIMEOUT, the kernels
  after the failed stage must leave unwritten data alone, and the next call on
  the same renderer must render correctly again.
* Allocation failure: a host-side hook refuses one device allocation as
  cudaMalloc does on an exhausted device; the call returns DL_E_OOM with the
  allocation in its message, and a later call succeeds.

The reference throws Error on device set-up failure (src/gpu/device.ts:29-35);
the C ABI returns the status and dl_last_error() holds the message, which the
Python mirror raises as DropletError."""
import numpy as np
import pytest

import droplet_b200 as dl
from droplet_b200 import _lib, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

L = _lib.load


@pytest.fixture(autouse=True)
def _clear_hooks():
    yield
    L().dl_test_withhold_status(0, 0)
    L().dl_test_set_wait_limit(0)
    L().dl_test_fail_allocation(-1)


@pytest.mark.parametrize("stage,tile", [(1, 1), (2, 1), (3, 1)], ids=["depth-sort", "emit", "pair-sort"])
def test_withheld_status_times_out_and_the_renderer_recovers(device, stage, tile):
    data = synth.plain_100k(60_000)
    cam = synth.pinhole(640, 360, (0.0, 0.0, 4.0))
    want = O.render(data, cam)["rgba"]
    r = dl.Renderer(device)
    assert np.array_equal(r.render(data, cam), want)
    L().dl_test_set_wait_limit(64)
    assert L().dl_test_withhold_status(stage, tile) == _lib.DL_OK
    with pytest.raises(dl.DropletError) as e:
        r.render(data, cam)
    assert e.value.code == _lib.DL_E_TIMEOUT and "timed out" in str(e.value)
    L().dl_test_withhold_status(0, 0)
    L().dl_test_set_wait_limit(0)
    assert np.array_equal(r.render(data, cam), want)        # same renderer, same buffers
    r.destroy()


def test_withheld_status_in_a_graph_replayed_batch(device):
    import torch
    data = synth.plain_100k(40_000)
    cams = synth.ring_cameras(4, radius=4.0, height=0.5, resolutions=[(320, 180), (480, 270)])
    r = dl.Renderer(device)
    stream = torch.cuda.Stream()
    r.set_stream(stream.cuda_stream)                 # a real stream: batches replay as CUDA graphs
    scene = r.upload(data, "f32")
    good = r.render_batch(scene, cams)
    L().dl_test_set_wait_limit(64)
    L().dl_test_withhold_status(2, 1)
    with pytest.raises(dl.DropletError) as e:
        r.render_batch(scene, cams)
    assert e.value.code == _lib.DL_E_TIMEOUT
    L().dl_test_withhold_status(0, 0)
    L().dl_test_set_wait_limit(0)
    again = r.render_batch(scene, cams)             # the hook is part of the graph's key: re-captured
    assert all(np.array_equal(a, b) for a, b in zip(good, again))
    scene.destroy()
    r.destroy()


def test_voxelize_wait_limit_default_and_tiny_limit_without_withholding(device):
    # a tiny limit with nothing withheld still completes (predecessors publish),
    # or reports a timeout; it never hangs and never returns wrong bits silently
    d = synth.voxel_1m(20_000)
    opts = {"voxelResolution": 0.1, "opacityCutoff": 0.1}
    ref = O.voxelize(d, 0.1, 0.1)
    L().dl_test_set_wait_limit(1)
    try:
        g = dl.voxelize(device, d, opts)
        assert np.array_equal(g.buffer.blockIdx, ref["block_idx"]) and np.array_equal(g.buffer.maskLo, ref["mask_lo"])
    except dl.DropletError as e:
        assert e.code == _lib.DL_E_TIMEOUT
    L().dl_test_set_wait_limit(0)
    g = dl.voxelize(device, d, opts)
    assert np.array_equal(g.buffer.blockIdx, ref["block_idx"]) and np.array_equal(g.buffer.maskHi, ref["mask_hi"])


@pytest.mark.parametrize("after", [0, 3, 9])
def test_refused_allocation_returns_oom_and_a_later_call_succeeds(device, after):
    data = synth.plain_100k(30_000)
    cam = synth.pinhole(480, 270, (0.0, 0.0, 4.0))
    want = O.render(data, cam)["rgba"]
    r = dl.Renderer(device)                          # fresh: its first frame allocates its buffers
    assert L().dl_test_fail_allocation(after) == _lib.DL_OK
    with pytest.raises(dl.DropletError) as e:
        r.render(data, cam)
    assert e.value.code == _lib.DL_E_OOM and "cudaMalloc" in str(e.value)
    assert np.array_equal(r.render(data, cam), want)   # the hook switched itself off
    r.destroy()


def test_refused_allocation_in_voxelize(device):
    d = synth.voxel_1m(10_000)
    dev2 = dl.createDevice()                         # a device handle with no voxel buffers yet
    L().dl_test_fail_allocation(0)
    with pytest.raises(dl.DropletError) as e:
        dl.voxelize(dev2, d, {"voxelResolution": 0.1, "opacityCutoff": 0.1})
    assert e.value.code == _lib.DL_E_OOM
    g = dl.voxelize(dev2, d, {"voxelResolution": 0.1, "opacityCutoff": 0.1})
    assert g.buffer.count > 0
    dev2.destroy()
