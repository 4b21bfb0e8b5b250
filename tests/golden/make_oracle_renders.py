"""Renders the converged oracle images the statistical GPU tests compare against.

    python tests/golden/make_oracle_renders.py [--threads N]

The oracle (the CPU restatement of the reference path tracer, oracle/) renders each scene at
4096 samples per pixel as 64 independent batches of 64 samples (seed 777, batch b taking
sample numbers 64 b .. 64 b + 63).  For every 16x16 pixel tile (the reference's tile size,
renderbuffer.hxx:45) the fixture keeps the tile mean over all batches and its standard
error from the spread of the 64 batch means (63 degrees of freedom), and for the 1/spp
test the means of 4x4 pixel blocks of the converged image.  Linear RGB, rows from the
bottom as the framebuffer stores them.  Output: tests/golden/oracle_renders.npz.

Scenes:
- cornell_box: the Cornell box of the first benchmark configuration, 256x256, max depth 10;
- cornell_box_medium: the same box filled with the homogeneous chromatic medium (sigma_s
  0.5 -> 2.0 per unit over the bins, sigma_a 0.1, Henyey-Greenstein g = 0.7), at 96x96
  instead of 1024x1024 to keep the oracle render within a minute, max depth 32.
"""
from __future__ import annotations

import argparse
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

BATCHES = 64
BATCH_SPP = 64
SEED = 777
TILE = 16
BLOCK = 4
SCENES = {"cornell_box": ((256, 256), 10), "cornell_box_medium": ((96, 96), 32)}


def block_means(img, xres, yres, b):
    a = img.reshape(yres, xres, 3)
    return a[: yres // b * b, : xres // b * b].reshape(yres // b, b, xres // b, b, 3).mean(axis=(1, 3))


def render(name, threads):
    from naivetrace_b200 import scenes
    from naivetrace_b200.scene import make_params
    from oracle.oracle import OracleScene, combine
    (xres, yres), depth = SCENES[name]
    scene = getattr(scenes, name)(xres, yres)
    o = OracleScene(scene, make_params(max_ray_depth=depth))
    npix = xres * yres
    tiles, total = [], np.zeros((npix, 3))
    for b in range(BATCHES):
        acc, light, splat = o.render(BATCH_SPP, seed=SEED, sample_offset=b * BATCH_SPP, nthreads=threads)
        img = combine(acc, light, BATCH_SPP, splat, npix).reshape(npix, 3)
        tiles.append(block_means(img, xres, yres, TILE))
        total += img
    tiles = np.stack(tiles)
    img = total / BATCHES
    return {
        f"{name}_tile_mean": tiles.mean(axis=0),
        f"{name}_tile_se": tiles.std(axis=0, ddof=1) / np.sqrt(BATCHES),
        f"{name}_block_mean": block_means(img, xres, yres, BLOCK).astype(np.float32),
        f"{name}_info": np.array([xres, yres, depth, BATCHES, BATCH_SPP, SEED], np.int64),
    }


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    a = ap.parse_args(argv)
    out = {}
    for name in SCENES:
        t0 = time.time()
        out.update(render(name, a.threads))
        print(f"{name}: {time.time() - t0:.0f} s")
    np.savez_compressed(HERE / "oracle_renders.npz", **out)
    print("wrote", HERE / "oracle_renders.npz")
    return 0


if __name__ == "__main__":
    sys.exit(main())
