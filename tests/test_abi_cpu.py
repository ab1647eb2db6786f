"""CPU tests of the C-ABI boundary: the library loads, exports every function
include/droplet_b200.h declares, and reports errors as the reference would
(a status + message, raised as an exception by the host API)."""
import ctypes
import os
import re

import numpy as np
import pytest

import droplet_b200 as dl
from droplet_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "droplet_b200.h")).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(dl_\w+)\(", src, re.M)))


def test_header_and_binding_agree():
    assert sorted(_lib.EXPORTS) == declared()


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, missing


def test_no_gpu_raises_like_reference(monkeypatch):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(dl.DropletError) as e:
        dl.createDevice()
    assert e.value.code == _lib.DL_E_NO_DEVICE


def test_null_arguments_are_rejected_without_a_device():
    L = _lib.load()
    assert L.dl_render(None, None, None, None, None, 0) == _lib.DL_E_INVALID_ARG
    assert "NULL" in L.dl_last_error().decode()
    assert L.dl_voxelize(None, None, None, None) == _lib.DL_E_INVALID_ARG
    # the block-mask buffer stages refuse a missing device before any device work
    bmin, dims = (ctypes.c_double * 3)(0.0, 0.0, 0.0), (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    assert L.dl_vox_query(None, None, None, None, 0, bmin, 0.1, dims, None, 0, None) == _lib.DL_E_INVALID_ARG
    assert "dl_vox_query" in L.dl_last_error().decode()
    n = ctypes.c_uint64(7)
    assert L.dl_vox_carve(None, None, None, None, 0, None, None, None, 0, None, None, None,
                          ctypes.byref(n)) == _lib.DL_E_INVALID_ARG
    assert "dl_vox_carve" in L.dl_last_error().decode()


def test_splatdata_validates_lengths():
    with pytest.raises(ValueError):
        dl.SplatData(2, np.zeros(5), np.zeros(8), np.zeros(6), np.zeros(2), np.zeros(6))
    with pytest.raises(ValueError):
        dl.SplatData(1, np.zeros(3), np.zeros(4), np.zeros(3), np.zeros(1), np.zeros(3), np.zeros(3), shBands=2)


def test_lookat_matches_reference_layout():
    m = dl.mat4LookAt((0, 0, 4), (0, 0, 0), (0, 1, 0))
    # math/index.ts:41-56: camera at +z looking at the origin -> identity rotation, translation -4
    assert np.allclose(m, [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, -4, 1])


def test_block_mask_buffer_semantics():
    b = dl.BlockMaskBuffer()
    b.addBlock(5, 1, 0)
    b.addBlock(5, 2, 0x80000000)
    b.addBlock(9, 0, 0)
    assert b.count == 1 and b.get(5).maskLo == 3 and b.get(5).maskHi == 0x80000000
    assert b.popcount() == 3 and b.get(9) is None


def test_morton_round_trip_and_bit_layout():
    """morton.ts:11-22: x, y, z bits interleaved x1 y1 z1 x2 y2 z2 from bit 0."""
    seen = set()
    for z in range(4):
        for y in range(4):
            for x in range(4):
                m = dl.mortonEncode3(x, y, z)
                assert dl.mortonDecode3(m) == (x, y, z)
                expect = sum(((v >> b) & 1) << (3 * b + a) for a, v in enumerate((x, y, z)) for b in range(2))
                assert m == expect
                seen.add(m)
    assert seen == set(range(64))
