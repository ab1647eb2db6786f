"""The learned tile-cost model: training data, training, persistence.

Data: per-tile features and measured rasterizer cost logged by the renderer
(DL_BATCH_LOG_TILES) from plain renders of seeded SH3 cluster scenes (seeds
3..10, 256 clusters in [-10, 10]^3, 40 ring views per seed over the four ring
resolutions and varying radius/height), about 2.2M tiles.  Target: log1p of
the measured cost (SM cycles / 16 summed over the tile's warps), standardised.
Training runs on the GPU through the library's own kernels (dl_mlp_train).
The trained parameters are stored in models/tile_cost_mlp.npz and loaded by
load_default(); with no file, scheduling falls back to launch order.

The block-cost model of the voxelizer is trained the same way on per-block
features and measured cost (SM cycles / 16 of vox_eval_k per 4x4x4 block)
logged from voxelizations of seeded 1M-Gaussian cluster scenes (seeds 3..10,
three resolutions, two cutoffs); models/voxel_block_cost_mlp.npz.

  python -m droplet_b200.learned [--splats N] [--epochs E] [--out PATH]
  python -m droplet_b200.learned --voxel [--epochs E] [--out PATH]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import _lib, synth
from .api import Mlp, Renderer, createDevice, voxelize

HERE = os.path.dirname(os.path.abspath(__file__))
MODEL_PATH = os.path.join(HERE, "models", "tile_cost_mlp.npz")
VOXEL_MODEL_PATH = os.path.join(HERE, "models", "voxel_block_cost_mlp.npz")
VOXEL_SETTINGS = ((0.04, 0.1), (0.05, 0.3), (0.07, 0.1))
TRAIN_SEEDS = tuple(range(3, 11))


def training_cameras(seed: int, count: int = 40):
    rng = np.random.default_rng(1000 + seed)
    cams = []
    for k in range(count):
        a = 2 * math.pi * k / count + rng.uniform(0, 0.1)
        radius = rng.uniform(8.0, 16.0)
        height = rng.uniform(-3.0, 5.0)
        w, h = synth.RING_RESOLUTIONS[k % len(synth.RING_RESOLUTIONS)]
        cams.append(synth.pinhole(w, h, (radius * math.sin(a), height, radius * math.cos(a))))
    return cams


HEADLINE_FLAGS = _lib.DL_BATCH_F16_RECORDS | _lib.DL_BATCH_FAST_EXP | _lib.DL_BATCH_CULL_OFFSCREEN


def collect(renderer: Renderer, seeds=TRAIN_SEEDS, splats: int = 3_000_000, views: int = 40, log=print,
            mode: str = "plain"):
    """Render every training view alone and log its tiles: the plain path
    (mode "plain") or the batched path's arithmetic and cull mode on an f16
    scene (mode "headline")."""
    import torch
    X, Y, S = [], [], []
    out = torch.empty(2560 * 1440 * 4, dtype=torch.uint8, device="cuda")
    flags = (_lib.DL_BATCH_PLAIN if mode == "plain" else HEADLINE_FLAGS) | _lib.DL_BATCH_LOG_TILES
    for seed in seeds:
        t = time.time()
        scene = renderer.upload(synth.sh3_3m(splats, seed=seed), "f32" if mode == "plain" else "f16")
        for cam in training_cameras(seed, views):
            renderer.render_batch(scene, [cam], flags=flags, outs=[out.data_ptr()])
            f, c = renderer.tile_log()
            X.append(f)
            Y.append(np.log1p(c))
            S.append(np.full(len(c), seed, np.int16))
        scene.destroy()
        log(f"seed {seed}: {sum(len(y) for y in Y)} tiles so far ({time.time() - t:.1f} s)")
    return np.concatenate(X), np.concatenate(Y).astype(np.float32), np.concatenate(S)


def voxel_scene(seed: int, n: int = 1_000_000):
    """A seeded 1M-Gaussian cluster scene drawn like the voxelize configuration."""
    return synth.cluster_scene(n, seed=seed, clusters=64, extent=5.0, log_lo=0.01, log_hi=0.1, op_mu=1.0,
                               op_sigma=1.5)


def collect_voxel(device, seeds=TRAIN_SEEDS, splats: int = 1_000_000, log=print):
    """Voxelize every training scene / setting and log its blocks."""
    X, Y, S = [], [], []
    for seed in seeds:
        t = time.time()
        d = voxel_scene(seed, splats)
        for res, cut in VOXEL_SETTINGS:
            f, c = voxelize(device, d, {"voxelResolution": res, "opacityCutoff": cut, "logBlocks": True}).blockLog
            X.append(f)
            Y.append(np.log1p(c))
            S.append(np.full(len(c), seed, np.int16))
        log(f"seed {seed}: {sum(len(y) for y in Y)} blocks so far ({time.time() - t:.1f} s)")
    return np.concatenate(X), np.concatenate(Y).astype(np.float32), np.concatenate(S)


def spearman(a, b) -> float:
    ra = np.argsort(np.argsort(a)).astype(np.float64)
    rb = np.argsort(np.argsort(b)).astype(np.float64)
    return float(np.corrcoef(ra, rb)[0, 1])


def train(mlp: Mlp, X, y, epochs: int = 8, batch: int = 8192, lr: float = 2e-3, seed: int = 0):
    mu, sd = float(y.mean()), float(y.std() + 1e-6)
    loss = mlp.train(X, (y - mu) / sd, epochs=epochs, batch=batch, lr=lr, seed=seed)
    return loss, mu, sd


def save(mlp: Mlp, path: str, meta: dict) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, params=mlp.get_params(), meta=json.dumps(meta))


def load(device, path: str = MODEL_PATH) -> Mlp:
    z = np.load(path)
    m = Mlp(device)
    m.set_params(z["params"])
    m.meta = json.loads(str(z["meta"]))
    return m


def load_default(device):
    return load(device, MODEL_PATH) if os.path.exists(MODEL_PATH) else None


def load_default_voxel(device):
    return load(device, VOXEL_MODEL_PATH) if os.path.exists(VOXEL_MODEL_PATH) else None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--splats", type=int, default=3_000_000)
    ap.add_argument("--views", type=int, default=40)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--out", default=None)
    ap.add_argument("--voxel", action="store_true", help="train the voxelizer's block-cost model")
    ap.add_argument("--mode", choices=("plain", "headline"), default="plain",
                    help="tile costs logged on the plain path or on the batched path's flags")
    a = ap.parse_args()
    dev = createDevice()
    t = time.time()
    if a.voxel:
        X, y, seeds = collect_voxel(dev)
        out = a.out or VOXEL_MODEL_PATH
    else:
        X, y, seeds = collect(Renderer(dev), splats=a.splats, views=a.views, mode=a.mode)
        out = a.out or MODEL_PATH
    t_collect = time.time() - t
    val = seeds == TRAIN_SEEDS[-1]                  # held-out seed for the prediction error
    mlp = Mlp(dev, seed=0)
    t = time.time()
    loss, mu, sd = train(mlp, X[~val], y[~val], epochs=a.epochs)
    t_train = time.time() - t
    pred = mlp.predict(X[val]) * sd + mu
    err = pred - y[val]
    meta = {"mode": "voxel" if a.voxel else a.mode, "samples": int(len(y)), "train_samples": int((~val).sum()), "val_seed": TRAIN_SEEDS[-1],
            "epochs": a.epochs, "final_loss": loss, "y_mean": mu, "y_std": sd,
            "val_rmse_log_cost": float(np.sqrt((err ** 2).mean())),
            "val_spearman": spearman(pred, y[val]),
            "val_r2": float(1 - (err ** 2).mean() / y[val].var()),
            "collect_s": t_collect, "train_s": t_train}
    save(mlp, out, meta)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
