"""Precision variants against the FP64 oracle, per scene configuration.

For each configuration and arithmetic variant the test reports, against the
oracle's FP64 pipeline (projection outputs and compositing in double): the
max and mean absolute error of the RGBA8 bytes in LSB (255 * colour), and the
share of pixels within +-1 LSB of the f32 oracle (the parity bar).  For the
exact f32 path it also reports the max / mean absolute error of the f32
colour accumulator against the f64 one.  Run with -s to see the table.
"""
import numpy as np
import pytest

import droplet_b200 as dl
from droplet_b200 import _lib, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

F16, FAST, F64D = _lib.DL_BATCH_F16_RECORDS, _lib.DL_BATCH_FAST_EXP, _lib.DL_BATCH_F64_DEGENERATE
VARIANTS = [("f32 records, exact exp", 0, "f32"),
            ("f32 + f64 degenerate conics", F64D, "f32"),
            ("f16 records", F16, "f32"),
            ("f16 records + f16 SH", F16, "f16"),
            ("f16 records + bf16 SH", F16, "bf16"),
            ("f16 records + f16 SH + ex2", F16 | FAST, "f16"),
            ("f16 + f16 SH + ex2 + f64 degenerate", F16 | FAST | F64D, "f16")]


def _configs():
    return [("cfg1 100k 1280x720", synth.plain_100k, lambda: [synth.plain_100k_camera()]),
            ("cfg3 3M SH3 1920x1080 + 2048x1024 equirect", synth.sh3_3m, synth.sh3_3m_cameras),
            ("cfg5 10M Zipf SH1 1920x1080", synth.zipf_10m, lambda: synth.zipf_10m_cameras(1))]


def _f64_bytes(acc64):
    """Composite over the default background (0, 0, 0, 1) in f64: bytes before rounding."""
    a = acc64.reshape(-1, 4)
    rgb = np.clip(a[:, :3], 0.0, 1.0) * 255.0
    alpha = np.clip(1.0 - a[:, 3] + a[:, 3] * 1.0, 0.0, 1.0) * 255.0
    return np.concatenate([rgb, alpha[:, None]], axis=1)


@pytest.mark.parametrize("cfg", range(3), ids=[c[0].split()[0] for c in _configs()])
def test_error_against_fp64_oracle(device, cfg):
    name, make, cams_fn = _configs()[cfg]
    data, cams = make(), cams_fn()
    r = dl.Renderer(device)
    scenes = {p: r.upload(data, p) for p in ("f32", "f16", "bf16")}
    lines = []
    for cam in cams:
        o = O.render(data, cam, f64=True, fields=("rgba", "accum", "accum64"))
        ref32 = o["rgba"].reshape(-1, 4).astype(np.int16)
        ref64 = _f64_bytes(o["accum64"])
        # f32 accumulator of the exact path against the f64 accumulator
        r.set_debug(True)
        r.render(data, cam)
        acc = r.debug_get("accum", np.float32)
        r.set_debug(False)
        acc_err = np.abs(acc.astype(np.float64) - o["accum64"])
        lines.append(f"{name} [{cam.projection} {cam.width}x{cam.height}] f32 accumulator vs f64: "
                     f"max {acc_err.max():.3e} mean {acc_err.mean():.3e}")
        # a sanity bound only (colours are unclamped sums here); the byte-level
        # bar below is the parity gate
        assert acc_err.max() < 5e-2 and acc_err.mean() < 1e-4
        for label, flags, prec in VARIANTS:
            got = r.render_batch(scenes[prec], [cam], flags=flags)[0].reshape(-1, 4)
            e64 = np.abs(got.astype(np.float64) - ref64)
            within = float((np.abs(got.astype(np.int16) - ref32).max(axis=1) <= 1).mean())
            lines.append(f"  {label:38s} vs f64: max {e64.max():6.3f} LSB mean {e64.mean():.4f} LSB; "
                         f"within 1 LSB of f32 oracle {within * 100:.3f}%")
            assert within >= 0.999, (label, within)
            if flags == 0 and prec == "f32":
                assert np.array_equal(got.astype(np.int16), ref32)      # exact path: bit-exact
    for s in scenes.values():
        s.destroy()
    r.destroy()
    print("\n" + "\n".join(lines))
