"""PLY loading (src/io/ply.ts): header rules, transforms, errors, round trip."""
import math
import struct

import numpy as np
import pytest

import droplet_b200 as dl
from droplet_b200 import ply, synth


def _ply(props, rows, fmt="binary_little_endian 1.0", extra_elements=""):
    head = f"ply\nformat {fmt}\nelement vertex {len(rows)}\n" + "".join(f"property float {p}\n" for p in props) + \
        extra_elements + "end_header\n"
    return head.encode() + b"".join(struct.pack("<" + "f" * len(r), *r) for r in rows)


BASE = ["x", "y", "z", "scale_0", "scale_1", "scale_2", "f_dc_0", "f_dc_1", "f_dc_2", "opacity",
        "rot_0", "rot_1", "rot_2", "rot_3"]


def _f32(v):
    return struct.unpack("<f", struct.pack("<f", v))[0]


def test_transforms_follow_the_reference_arithmetic():
    row = [1.5, -2.25, 3.0, -3.0, -2.5, -2.0, 0.7, -0.3, 1.1, 0.25, 2.0, 1.0, -1.0, 0.5]
    for flip in (True, False):
        d = ply.loadPlySplats(_ply(BASE, [row]), {"flipY": flip})
        s = -1.0 if flip else 1.0
        assert d.count == 1 and d.shBands == 0 and d.colorsSH is None
        assert list(d.positions) == [1.5, s * -2.25, 3.0]
        assert list(d.logScales) == [-3.0, -2.5, -2.0] and list(d.opacityLogits) == [0.25]
        c0 = 0.28209479177387814
        assert list(d.colorsDC) == [_f32(c0 * _f32(0.7)), _f32(c0 * _f32(-0.3)), _f32(c0 * _f32(1.1))]
        n = math.sqrt(4 + 1 + 1 + 0.25)
        assert list(d.rotations) == [_f32(2 / n), _f32(s * 1 / n), _f32(-1 / n), _f32(s * 0.5 / n)]


def test_property_order_and_sh_bands_are_read_by_name():
    rng = np.random.default_rng(3)
    for bands, k in ((1, 9), (2, 24), (3, 45)):
        props = BASE + [f"f_rest_{i}" for i in range(k)]
        perm = rng.permutation(len(props))
        rows = rng.normal(size=(5, len(props))).astype(np.float32)
        d = ply.loadPlySplats(_ply([props[i] for i in perm], rows[:, perm].tolist()), {"flipY": False})
        assert d.shBands == bands
        assert np.array_equal(d.colorsSH.reshape(5, k), rows[:, 14:])
        assert np.array_equal(d.positions.reshape(5, 3), rows[:, :3])


def test_too_few_f_rest_are_ignored_like_the_reference():
    d = ply.loadPlySplats(_ply(BASE + ["f_rest_0", "f_rest_1"], [[0.0] * 16]))
    assert d.shBands == 0 and d.colorsSH is None


def test_zero_quaternion_and_other_elements():
    row = [0.0] * 10 + [0.0, 0.0, 0.0, 0.0]
    faces = "element face 0\nproperty list uchar int vertex_indices\n"
    d = ply.loadPlySplats(_ply(BASE, [row], extra_elements=faces))
    assert list(d.rotations) == [0.0, -0.0, 0.0, -0.0]           # || 1: divided by 1


def test_nan_and_infinite_quaternions_follow_math_hypot():
    # Math.hypot(w, x, y, z) || 1: a NaN component gives NaN -> 1 (the finite
    # components pass through); an infinite one gives +Infinity even beside a NaN
    nan, inf = float("nan"), float("inf")
    rows = [[0.0] * 10 + [nan, 0.5, 0.25, 2.0], [0.0] * 10 + [inf, nan, 1.0, 2.0]]
    d = ply.loadPlySplats(_ply(BASE, rows), {"flipY": False})
    q = d.rotations.reshape(-1, 4)
    assert np.isnan(q[0, 0]) and list(q[0, 1:]) == [0.5, 0.25, 2.0]
    assert np.isnan(q[1, 0]) and np.isnan(q[1, 1]) and list(q[1, 2:]) == [0.0, 0.0]


@pytest.mark.parametrize("make,msg", [
    (lambda: b"ply\nformat binary_little_endian 1.0\nelement vertex 1\n", "end_header not found"),
    (lambda: b"plx\nend_header\n", "missing magic"),
    (lambda: _ply(BASE, [[0.0] * 14], fmt="ascii 1.0"), "ASCII PLY not supported"),
    (lambda: _ply(BASE, [[0.0] * 14], fmt="binary_big_endian 1.0"), "only little-endian"),
    (lambda: _ply(BASE, []), "no vertices"),
    (lambda: _ply(BASE, [[0.0] * 14])[:-4], "data section truncated"),
    (lambda: _ply(BASE[:-1], [[0.0] * 13]), 'missing property "rot_3"'),
    (lambda: _ply(BASE + [f"f_rest_{k}" for k in range(12)], [[0.0] * 26]), "no SH band layout"),
    (lambda: _ply(BASE, [[0.0] * 14]).replace(b"property float opacity", b"property uchar opacity"),
     "mixed property types"),
    (lambda: _ply(BASE, [[0.0] * 14]).replace(b"property float opacity", b"property double opacity"),
     'unsupported property type "double"'),
])
def test_errors_match_the_reference(make, msg):
    with pytest.raises(ValueError, match=msg):
        ply.loadPlySplats(make())


def test_round_trip_and_bounds(tmp_path):
    d = synth.cluster_scene(2000, seed=5, clusters=4, extent=3.0, bands=3)
    path = str(tmp_path / "s.ply")
    ply.savePlySplats(d, path)
    e = ply.loadPlySplats(path)
    assert e.count == d.count and e.shBands == 3
    assert np.array_equal(e.positions, d.positions) and np.array_equal(e.logScales, d.logScales)
    assert np.array_equal(e.colorsSH, d.colorsSH) and np.array_equal(e.opacityLogits, d.opacityLogits)
    assert np.allclose(e.colorsDC, d.colorsDC, rtol=1e-6, atol=1e-7)
    assert np.allclose(e.rotations, d.rotations, rtol=1e-6, atol=1e-7)
    b = ply.splatBounds(e)
    p = d.positions.reshape(-1, 3)
    assert b["min"] == [float(v) for v in p.min(0)] and b["max"] == [float(v) for v in p.max(0)]
    assert dl.loadPlySplats is ply.loadPlySplats


# ---- the C-ABI loader (dl_ply_load) against the Python loader, ordinary host memory
def _native(buf, opts=None):
    return dl.PlySplats(buf, opts, pinned=False)


def _same(a, b):
    assert a.count == b.count and a.shBands == b.shBands
    for k in ("positions", "rotations", "logScales", "opacityLogits", "colorsDC", "colorsSH"):
        x, y = getattr(a, k), getattr(b, k)
        if x is None or y is None:
            assert x is None and y is None, k
        else:
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), k


def test_native_loader_matches_the_python_loader():
    rng = np.random.default_rng(11)
    for bands, k in ((0, 0), (1, 9), (2, 24), (3, 45)):
        props = BASE + [f"f_rest_{i}" for i in range(k)]
        perm = rng.permutation(len(props))
        rows = rng.normal(size=(257, len(props))).astype(np.float32)
        rows[3, 10:14] = 0.0                                   # zero quaternion
        rows[4, 10] = np.nan                                   # NaN component
        rows[5, 11] = np.inf                                   # infinite component
        buf = _ply([props[i] for i in perm], rows[:, perm].tolist(),
                   extra_elements="element face 0\nproperty list uchar int vertex_indices\n")
        for flip in (True, False):
            p = _native(buf, {"flipY": flip})
            _same(p.data, ply.loadPlySplats(buf, {"flipY": flip}))
            p.destroy()


def test_native_loader_reads_unaligned_data_and_files(tmp_path):
    d = synth.cluster_scene(500, seed=6, clusters=3, extent=2.0, bands=2)
    path = str(tmp_path / "s.ply")
    ply.savePlySplats(d, path)
    raw = open(path, "rb").read()
    _same(_native(path).data, ply.loadPlySplats(path))
    head = raw.index(b"end_header\n")
    shifted = raw[:head] + b" " + raw[head:]                  # one header byte more: data at an odd offset
    _same(_native(shifted).data, ply.loadPlySplats(shifted))


@pytest.mark.parametrize("make,msg", [
    (lambda: b"ply\nformat binary_little_endian 1.0\nelement vertex 1\n", "end_header not found"),
    (lambda: b"plx\nend_header\n", "missing magic"),
    (lambda: _ply(BASE, [[0.0] * 14], fmt="ascii 1.0"), "ASCII PLY not supported"),
    (lambda: _ply(BASE, [[0.0] * 14], fmt="binary_big_endian 1.0"), "only little-endian"),
    (lambda: _ply(BASE, []), "no vertices"),
    (lambda: _ply(BASE, [[0.0] * 14])[:-4], "data section truncated"),
    (lambda: _ply(BASE[:-1], [[0.0] * 13]), 'missing property "rot_3"'),
    (lambda: _ply(BASE + [f"f_rest_{k}" for k in range(12)], [[0.0] * 26]), "no SH band layout"),
    (lambda: _ply(BASE, [[0.0] * 14]).replace(b"property float opacity", b"property uchar opacity"),
     "mixed property types"),
    (lambda: _ply(BASE, [[0.0] * 14]).replace(b"property float opacity", b"property double opacity"),
     'unsupported property type "double"'),
])
def test_native_loader_errors_match(make, msg):
    with pytest.raises(ValueError, match=msg) as e:
        _native(make())
    with pytest.raises(ValueError) as f:
        ply.loadPlySplats(make())
    assert str(e.value) == str(f.value)
