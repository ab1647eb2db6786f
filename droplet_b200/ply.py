"""3DGS PLY loading: loadPlySplats and splatBounds (src/io/ply.ts:1-255).

Same accepted layouts, transforms and errors as the reference loader:
binary little-endian PLY only, a `vertex` element whose properties are all
`float` (any order: fields are found by name), `f_dc_*` scaled by
SH_C0 = 1/(2 sqrt(pi)) into the "(colour - 0.5)" convention, quaternions
(rot_0..3 = w, x, y, z) normalized, optional `f_rest_*` SH in channel-major
order, and `flipY` (default true) negating y and the quaternion's x and z.
The arithmetic follows the reference: products and quotients in float64 (JS
numbers) rounded once to float32.  The reference normalizes with Math.hypot;
here the norm is sqrt of the float64 sum of squares, which can differ from
hypot in the last float64 ulp only, below the float32 rounding that follows.

One deliberate difference: an `f_rest_*` count that is not 0, 9, 24 or 45 (no
SH band layout) raises ValueError; the reference would return an SH array
whose per-splat stride disagrees with its shBands.
"""
from __future__ import annotations

import re
from typing import Optional, Union

import numpy as np

from .types import SplatData, numSHCoeffsPerChannel

SH_C0 = 0.28209479177387814            # ply.ts:23
_HEADER_MAX = 65536                     # ply.ts:45
_SIZE = {"float": 4, "uchar": 1, "int": 4}


def _parse_header(data: bytes):
    """ply.ts:41-92."""
    head = data[:_HEADER_MAX]
    end = head.find(b"end_header\n")
    if end < 0:
        raise ValueError("PLY: end_header not found in first 64KB")
    offset = end + len(b"end_header\n")
    lines = [ln.strip() for ln in head[:end].decode("utf-8", errors="replace").split("\n")]
    lines = [ln for ln in lines if ln]
    if not lines or lines[0] != "ply":
        raise ValueError("PLY: missing magic")
    count, binary, little, props, in_vertex = 0, False, True, [], False
    for line in lines[1:]:
        if line.startswith("format "):
            binary = "binary" in line
            little = "little_endian" in line
            continue
        if line.startswith("element vertex "):
            m = re.match(r"\s*([+-]?\d+)", line[len("element vertex "):])   # parseInt: leading digits
            count = int(m.group(1)) if m else -1
            in_vertex = True
            continue
        if line.startswith("element "):
            in_vertex = False
            continue
        if in_vertex and line.startswith("property "):
            parts = line.split()
            t = parts[1] if len(parts) > 1 else ""
            name = parts[2] if len(parts) > 2 else ""
            if t not in _SIZE:
                raise ValueError(f'PLY: unsupported property type "{t}"')
            props.append((t, name))
    if not binary:
        raise ValueError("PLY: ASCII PLY not supported (binary only)")
    if not little:
        raise ValueError("PLY: only little-endian supported")
    if count <= 0:
        raise ValueError("PLY: no vertices")
    return count, props, offset


def loadPlySplats(source: Union[bytes, bytearray, memoryview, str], opts: Optional[dict] = None) -> SplatData:
    """ply.ts:120-239.  source: the file's bytes, or a path.  opts: {flipY=True}."""
    if isinstance(source, str):
        with open(source, "rb") as f:
            source = f.read()
    data = bytes(source) if not isinstance(source, bytes) else source
    flip = True if not opts or opts.get("flipY") is None else bool(opts["flipY"])
    count, props, offset = _parse_header(data)
    idx = {}
    for p, (_, name) in enumerate(props):
        idx[name] = p                      # a repeated name keeps its last index, as the reference's map
    if not all(t == "float" for t, _ in props):
        raise ValueError("PLY: mixed property types not yet supported")
    per = len(props)
    total = count * per * 4
    if offset + total > len(data):
        raise ValueError(f"PLY: data section truncated (need {total} bytes, have {len(data) - offset})")
    flat = np.frombuffer(data, dtype="<f4", count=count * per, offset=offset).reshape(count, per)

    def need(n):
        if n not in idx:
            raise ValueError(f'PLY: missing property "{n}"')
        return idx[n]

    def col(n):
        return flat[:, need(n)].astype(np.float64)

    k_rest = 0
    while f"f_rest_{k_rest}" in idx:
        k_rest += 1
    cpc = k_rest // 3
    bands = 3 if cpc >= 15 else 2 if cpc >= 8 else 1 if cpc >= 3 else 0
    if bands and cpc != numSHCoeffsPerChannel(bands):
        raise ValueError(f"PLY: {k_rest} f_rest properties match no SH band layout (9, 24 or 45)")

    y_sign = -1.0 if flip else 1.0
    x, y, z = col("x"), col("y"), col("z")
    positions = np.stack([x, y_sign * y, z], axis=1).astype(np.float32)
    log_scales = np.stack([col("scale_0"), col("scale_1"), col("scale_2")], axis=1).astype(np.float32)
    opacity = col("opacity").astype(np.float32)
    dc = np.stack([SH_C0 * col("f_dc_0"), SH_C0 * col("f_dc_1"), SH_C0 * col("f_dc_2")], axis=1).astype(np.float32)
    w, qx, qy, qz = col("rot_0"), col("rot_1"), col("rot_2"), col("rot_3")
    # Math.hypot(...) || 1: hypot is +Infinity when any argument is infinite
    # (even beside a NaN), NaN when one is NaN, and `|| 1` maps both NaN and 0 to 1
    with np.errstate(invalid="ignore", over="ignore"):
        n = np.sqrt(w * w + qx * qx + qy * qy + qz * qz)
    n = np.where(np.isinf(w) | np.isinf(qx) | np.isinf(qy) | np.isinf(qz), np.inf, n)
    n = np.where(np.isnan(n) | (n == 0.0), 1.0, n)
    f = -1.0 if flip else 1.0
    rotations = np.stack([w / n, (f * qx) / n, qy / n, (f * qz) / n], axis=1).astype(np.float32)
    sh = None
    if bands:
        sh = np.ascontiguousarray(np.stack([flat[:, idx[f"f_rest_{k}"]] for k in range(3 * cpc)], axis=1),
                                  dtype=np.float32)
    return SplatData(count, positions, rotations, log_scales, opacity, dc, sh, bands)


def splatBounds(data: SplatData):
    """ply.ts:242-255 — axis-aligned bounds of the splat centres."""
    p = data.positions.reshape(-1, 3)
    if p.shape[0] == 0:
        inf = float("inf")
        return {"min": [inf, inf, inf], "max": [-inf, -inf, -inf]}
    return {"min": [float(v) for v in p.min(axis=0)], "max": [float(v) for v in p.max(axis=0)]}


def savePlySplats(data: SplatData, path: Optional[str] = None, flipY: bool = True) -> bytes:
    """Write SplatData as a binary little-endian 3DGS PLY that loadPlySplats
    reads back to the same arrays (up to float32 rounding of the inverse
    transforms).  Not part of the reference; used to make test files."""
    n = data.count
    m = numSHCoeffsPerChannel(data.shBands)
    names = ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2"] + [f"f_rest_{k}" for k in range(3 * m)] + \
            ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]
    s = -1.0 if flipY else 1.0
    pos = data.positions.reshape(n, 3).astype(np.float64)
    rot = data.rotations.reshape(n, 4).astype(np.float64)
    cols = [pos[:, 0], s * pos[:, 1], pos[:, 2]] + list((data.colorsDC.reshape(n, 3).astype(np.float64) / SH_C0).T)
    if m:
        cols += list(data.colorsSH.reshape(n, 3 * m).T)
    cols += [data.opacityLogits] + list(data.logScales.reshape(n, 3).T) + \
            [rot[:, 0], s * rot[:, 1], rot[:, 2], s * rot[:, 3]]
    body = np.stack([np.asarray(c, np.float64) for c in cols], axis=1).astype("<f4").tobytes()
    head = "ply\nformat binary_little_endian 1.0\n" + f"element vertex {n}\n" + \
           "".join(f"property float {nm}\n" for nm in names) + "end_header\n"
    out = head.encode() + body
    if path:
        with open(path, "wb") as f:
            f.write(out)
    return out
