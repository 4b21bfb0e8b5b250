"""Participating media on the GPU against the oracle: homogeneous media bounded by
volume-boundary meshes, a medium entered through a glass surface, overlapping media with
priorities, absorbing-only media, the camera inside a medium, and the three phase
functions (GPU).

The random numbers are consumed in the same order on both sides (next-event estimation,
scatter sample, spectral tracking, emission, Russian roulette per vertex), so per-path
parity holds here as it does for surfaces, apart from paths whose tracking or
roulette decision flips under float rounding.
"""
import numpy as np
import pytest

from naivetrace_b200 import abi, scenes
from naivetrace_b200.algo import GpuContext
from naivetrace_b200.scene import make_params
from oracle.oracle import OracleScene, combine
from test_gpu_render import render_both, tile_means

pytestmark = pytest.mark.gpu

MEDIA_SCENES = ["cornell_box_medium", "cornell_box_media_mix"]


@pytest.mark.parametrize("name", MEDIA_SCENES)
def test_media_per_path_parity(gpu_lib, name):
    scene = getattr(scenes, name)(32, 32)
    (ag, lg, sg), (ao, lo, so), g, o = render_both(scene, 4, 10)
    assert sg == so
    ag = ag.reshape(-1, 3)
    ao = ao.reshape(-1, 3)
    scale = max(np.abs(ao).mean(), 1e-6)
    close = np.all(np.abs(ag - ao) <= 1e-3 * np.abs(ao) + 1e-3 * scale, axis=1)
    assert close.mean() >= 0.95, close.mean()
    np.testing.assert_allclose(ag[close].sum(axis=0), ao[close].sum(axis=0), rtol=1e-3)
    np.testing.assert_allclose(lg.sum(), lo.sum(), rtol=0.05, atol=1e-6)
    assert g.stats()["error_flags"] == 0


@pytest.mark.parametrize("name", MEDIA_SCENES)
def test_media_tile_z_test(gpu_lib, name):
    """16x16 tile means of independent GPU and oracle renders: at least 97 % of the
    tile-channels within 3 sigma, all within 4 sigma (as for surfaces)."""
    xres = yres = 64
    scene = getattr(scenes, name)(xres, yres)
    p = make_params(max_ray_depth=10)
    g = GpuContext(scene, p)
    o = OracleScene(scene, p)
    K, spp = 32, 16
    tg, to = [], []
    for k in range(K):
        g.clear()
        g.render(spp, seed=100 + k)
        acc, light, sppc, splat = g.accumulators()
        tg.append(tile_means(combine(acc, light, spp, splat, g.npix), xres, yres))
        acc_o, light_o, splat_o = o.render(spp, seed=500 + k)
        to.append(tile_means(combine(acc_o, light_o, spp, splat_o, o.npix), xres, yres))
    tg, to = np.array(tg), np.array(to)
    mg, mo = tg.mean(0), to.mean(0)
    se = np.sqrt(tg.var(0, ddof=1) / K + to.var(0, ddof=1) / K)
    z = np.abs(mg - mo) / np.maximum(se, 1e-12)
    assert (z < 3.0).mean() >= 0.97, (z < 3.0).mean()
    assert np.all(z < 4.0), z.max()


def test_media_sample_modes_agree(gpu_lib):
    """BSDF-only, light-only and MIS estimates converge to the same image in a medium."""
    scene = scenes.cornell_box_medium(16, 16)
    means = []
    for mode in (abi.SAMPLE_BOTH, abi.SAMPLE_BSDF, abi.SAMPLE_LIGHTS):
        g = GpuContext(scene, make_params(max_ray_depth=10, pt_sample_mode=mode))
        g.render(4096, seed=5)
        means.append(g.framebuffer().reshape(-1, 3).mean(axis=0))
    np.testing.assert_allclose(means[1], means[0], rtol=0.03)
    np.testing.assert_allclose(means[2], means[0], rtol=0.03)


def test_media_change_the_image(gpu_lib):
    """Seen through the medium the area light is attenuated (its pixels lose most of their
    radiance), and the pass runs the medium-tracking launches."""
    a = GpuContext(scenes.cornell_box(32, 32), make_params(max_ray_depth=10))
    a.render(256, seed=3)
    b = GpuContext(scenes.cornell_box_medium(32, 32), make_params(max_ray_depth=10))
    b.render(256, seed=3)
    ia, ib = a.framebuffer().reshape(-1, 3).sum(1), b.framebuffer().reshape(-1, 3).sum(1)
    light = ia > 20 * np.median(ia)
    assert light.sum() > 0
    # Extinction 0.6 .. 2.1 per unit over about 0.7 units of medium (the camera is outside
    # the medium box), partly made up by light scattered into the view ray.
    assert ib[light].mean() < 0.85 * ia[light].mean()
    assert b.stats()["kernel_launches"] > a.stats()["kernel_launches"]
