"""dl_render_static: the render path for callers that may not allocate GPU memory.

Some hosts own the whole device through their own allocator (an engine or a
framework that reserves GPU memory up front and forbids foreign cudaMalloc),
or run a real-time loop that must not allocate once started.  For them the
library offers dl_render_static, which takes all its device scratch from one
fixed array reserved when the library is loaded.  These tests call it through
the C ABI and require the very same RGBA8 bytes as dl_render (the tolerance
the render parity tests use: bit-exact), on two calls in a row with different
scenes so that anything the first call leaves in the shared array cannot leak
into the second.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

import droplet_b200 as dl
from droplet_b200 import _lib, synth
from droplet_b200.api import _bg, _camera, _splats

pytestmark = pytest.mark.gpu


def render_static(data, cam, bg=(0.0, 0.0, 0.0, 1.0), max_cov=0):
    out = np.empty(cam.width * cam.height * 4, np.uint8)
    st = _lib.load().dl_render_static(ctypes.byref(_splats(data)), ctypes.byref(_camera(cam)), _bg(bg), max_cov,
                                      out.ctypes.data, out.size)
    return st, out


def test_static_render_matches_dl_render_twice():
    dev = dl.createDevice()
    r = dl.Renderer(dev)
    cases = [(synth.cluster_scene(16_000, seed=41, clusters=16, extent=1.5, bands=3),
              synth.pinhole(1280, 720, (0.0, 0.5, 4.0)), (0.0, 0.0, 0.0, 1.0)),
             (synth.plain_100k(5_000), synth.pinhole(640, 360, (0.3, 0.0, 3.0)), (0.2, 0.1, 0.0, 0.5))]
    for data, cam, bg in cases:                     # two calls in a row
        want = r.render(data, cam, bg)
        st, got = render_static(data, cam, bg)
        assert st == _lib.DL_OK, _lib.load().dl_last_error().decode()
        assert np.array_equal(got, want)
    r.destroy()


def test_static_render_allocates_nothing():
    # after one warm-up call (driver set-up such as pageable-copy staging), the
    # device's free memory must not move across further calls
    import torch
    data = synth.cluster_scene(12_000, seed=43, clusters=8, extent=1.5, bands=1)
    cam = synth.pinhole(960, 540, (0.0, 0.3, 4.0))
    st, first = render_static(data, cam)
    assert st == _lib.DL_OK, _lib.load().dl_last_error().decode()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        st, again = render_static(data, cam)
        assert st == _lib.DL_OK and np.array_equal(again, first)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_static_render_rejects_sizes_beyond_its_array():
    data = synth.plain_100k(16_385)
    st, _ = render_static(data, synth.pinhole(320, 180, (0.0, 0.0, 4.0)))
    assert st == _lib.DL_E_CAPACITY
    assert "16384" in _lib.load().dl_last_error().decode()
    st, _ = render_static(synth.plain_100k(100), synth.pinhole(1920, 1080, (0.0, 0.0, 4.0)))
    assert st == _lib.DL_E_CAPACITY
    # within the splat and pixel limits, but large splats bin to more tile
    # pairs than the array holds (2000 splats x ~3600 tiles of a 1280x720 view)
    n = 2000
    rng = np.random.default_rng(5)
    big = dl.SplatData(n, (rng.random((n, 3)) * 0.2 - 0.1).astype(np.float32),
                       np.tile(np.array([1, 0, 0, 0], np.float32), (n, 1)), np.full((n, 3), np.log(0.6), np.float32),
                       np.full(n, 2.0, np.float32), np.full((n, 3), 0.3, np.float32))
    st, _ = render_static(big, synth.pinhole(1280, 720, (0.0, 0.0, 3.0)))
    assert st == _lib.DL_E_CAPACITY
    assert "tile pairs" in _lib.load().dl_last_error().decode()
    # and the next call in range still renders correctly
    data = synth.plain_100k(3_000)
    cam = synth.pinhole(640, 360, (0.0, 0.0, 4.0))
    st, got = render_static(data, cam)
    assert st == _lib.DL_OK
    r = dl.Renderer(dl.createDevice())
    assert np.array_equal(got, r.render(data, cam))
    r.destroy()
