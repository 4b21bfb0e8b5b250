"""Statistical oracle at the configurations' sizes (GPU): the CUDA tracer's images against
converged 4096-spp renders of the CPU oracle (tests/golden/oracle_renders.npz, made by
tests/golden/make_oracle_renders.py).

1. Tile z-test: every 16x16 tile mean of the GPU image, per RGB channel, lies within the
   Bonferroni-corrected bound of the oracle's: z = (GPU mean - oracle mean) / sqrt(se_gpu^2 +
   se_oracle^2), each standard error from 64 independent batches (63 degrees of freedom).
   The family of T = tiles x 3 tests is held to a 1 % false-alarm rate, so each |z| must
   stay below the two-sided Student-t quantile at 0.01 / T (about 4.8 for the 768 tests of
   the 256x256 Cornell box).  In addition the number of tests beyond 3 sigma stays within
   the 99.9 % quantile of its binomial distribution (about 9 of 768, 3 of 108).
2. relMSE = mean((I - R)^2 / (R^2 + 1e-2)) over 4x4 pixel blocks against the oracle's
   converged blocks falls as 1/spp from 4 to 256 spp.
"""
from pathlib import Path

import numpy as np
import pytest
from scipy import stats

from naivetrace_b200 import scenes
from naivetrace_b200.algo import GpuContext
from naivetrace_b200.scene import make_params

pytestmark = pytest.mark.gpu

FIXTURE = Path(__file__).resolve().parent / "golden" / "oracle_renders.npz"
FAMILY_ALPHA = 0.01


@pytest.fixture(scope="module")
def oracle_renders():
    return dict(np.load(FIXTURE))


def block_means(img, xres, yres, b):
    a = img.reshape(yres, xres, 3)
    return a[: yres // b * b, : xres // b * b].reshape(yres // b, b, xres // b, b, 3).mean(axis=(1, 3))


@pytest.mark.parametrize("name,spp", [("cornell_box", 16), ("cornell_box_medium", 16)])
def test_tiles_against_converged_oracle(gpu_lib, oracle_renders, name, spp):
    xres, yres, depth, batches, _, _ = oracle_renders[f"{name}_info"]
    om, ose = oracle_renders[f"{name}_tile_mean"], oracle_renders[f"{name}_tile_se"]
    g = GpuContext(getattr(scenes, name)(int(xres), int(yres)), make_params(max_ray_depth=int(depth)))
    tiles = []
    for b in range(int(batches)):
        g.clear()
        g.render(spp, seed=4242 + b)
        tiles.append(block_means(g.framebuffer().astype(np.float64), int(xres), int(yres), 16))
    tiles = np.stack(tiles)
    gm = tiles.mean(axis=0)
    gse = tiles.std(axis=0, ddof=1) / np.sqrt(len(tiles))
    se = np.sqrt(gse ** 2 + ose ** 2)
    z = np.where(se > 0, np.abs(gm - om) / np.maximum(se, 1e-300), 0.0)
    tests = z.size
    bound = stats.t.ppf(1.0 - FAMILY_ALPHA / (2 * tests), df=int(batches) - 1)
    assert z.max() < bound, (z.max(), bound, np.unravel_index(z.argmax(), z.shape))
    p3 = 2 * stats.t.sf(3.0, df=int(batches) - 1)
    assert (z >= 3.0).sum() <= stats.binom.ppf(0.999, tests, p3), ((z >= 3.0).sum(), tests)


def test_relmse_against_converged_oracle_falls_as_one_over_spp(gpu_lib, oracle_renders):
    xres, yres, depth = (int(x) for x in oracle_renders["cornell_box_info"][:3])
    R = oracle_renders["cornell_box_block_mean"].astype(np.float64)
    scene = scenes.cornell_box(xres, yres)
    p = make_params(max_ray_depth=depth)
    spps = [4, 16, 64, 256]
    errs = []
    for spp in spps:
        vals = []
        for k in range(4):
            g = GpuContext(scene, p)
            g.render(spp, seed=9000 + 10 * spp + k)
            I = block_means(g.framebuffer().astype(np.float64), xres, yres, 4)
            vals.append(np.mean((I - R) ** 2 / (R * R + 1e-2)))
            g.close()
        errs.append(np.mean(vals))
    ratios = [errs[i] / errs[i + 1] for i in range(len(errs) - 1)]
    for r in ratios:
        assert 3.0 < r < 5.3, (errs, ratios)
    # spp x relMSE stays constant within the spread of four renders per point
    prod = np.array(errs) * np.array(spps)
    assert prod.max() / prod.min() < 1.4, prod
