"""The null-path tracer (--algo pt2) on the GPU against the CPU oracle (GPU).

1. Per-path parity: the device and the oracle run the same PCG32 stream per camera sample
   (tracking, light pick, light sample, BSDF sample in the same order; the shadow ray's
   transmission on a stream seeded from the path state at the connection), so at a few
   samples per pixel the accumulators agree pixel by pixel up to float rounding, apart from
   the paths whose tracking or reflect/refract decision flips under it.  Scenes cover
   diffuse, glass after a rough bounce (the mollified dielectric), microfacet, mirror,
   spheres, an environment map with a sun, homogeneous media behind glass and overlapping
   media with priorities.
2. Statistical parity: tile means of independent renders in a media scene (z-test).
3. pt2 against pt on the GPU in BSDF-only mode (same vertices collect emission at depths
   D + 1 and D).
4. Quasi-random sampling (qmc): per-path parity over two passes, lower error than PCG32.
5. The rest of the interface: multi-view batches, rejected combinations.
"""
import copy

import numpy as np
import pytest

from naivetrace_b200 import abi, scenes
from naivetrace_b200.algo import GpuContext
from naivetrace_b200.scene import make_params
from oracle.oracle import OracleScene, combine
from test_gpu_render import tile_means

pytestmark = pytest.mark.gpu


def _render_both(scene, spp, depth, seed=1, mode=abi.SAMPLE_BOTH):
    p = make_params(max_ray_depth=depth, pt_sample_mode=mode, algo=abi.ALGO_PT2)
    g = GpuContext(scene, p)
    g.render(spp, seed)
    acc_g, light_g, _, splat_g = g.accumulators()
    o = OracleScene(scene, p)
    acc_o, light_o, splat_o = o.render(spp, seed=seed)
    return acc_g.reshape(-1, 3), acc_o.reshape(-1, 3), light_g, g


@pytest.mark.parametrize("name,depth,frac", [
    ("cornell_box", 10, 0.97), ("cornell_box_materials", 10, 0.95), ("spheres_box", 10, 0.93),
    ("terrain_spheres_small", 12, 0.97), ("cornell_box_medium", 10, 0.93), ("cornell_box_media_mix", 10, 0.93)])
def test_pt2_per_path_parity(gpu_lib, name, depth, frac):
    scene = getattr(scenes, name)(32, 32) if name != "terrain_spheres_small" else scenes.terrain_spheres_small(48, 27)
    ag, ao, lg, g = _render_both(scene, 4, depth)
    assert g.stats()["error_flags"] == 0
    assert np.all(lg == 0)
    scale = max(np.abs(ao).mean(), 1e-6)
    close = np.all(np.abs(ag - ao) <= 1e-3 * np.abs(ao) + 1e-3 * scale, axis=1)
    assert close.mean() >= frac, close.mean()
    np.testing.assert_allclose(ag[close].sum(axis=0), ao[close].sum(axis=0), rtol=1e-3)


@pytest.mark.parametrize("mode", [abi.SAMPLE_BSDF, abi.SAMPLE_LIGHTS])
def test_pt2_per_path_parity_modes(gpu_lib, mode):
    scene = scenes.cornell_box_medium(32, 32)
    ag, ao, _, g = _render_both(scene, 4, 8, mode=mode)
    scale = max(np.abs(ao).mean(), 1e-6)
    close = np.all(np.abs(ag - ao) <= 1e-3 * np.abs(ao) + 1e-3 * scale, axis=1)
    assert close.mean() >= 0.93, close.mean()


@pytest.mark.parametrize("name", ["cornell_box_media_mix", "cornell_box_materials"])
def test_pt2_tile_z_test(gpu_lib, name):
    """16x16 tile means of independent GPU and oracle renders: at least 97 % of the
    tile-channels within 3 sigma, all within 4 sigma."""
    xres = yres = 64
    scene = getattr(scenes, name)(xres, yres)
    p = make_params(max_ray_depth=10, algo=abi.ALGO_PT2)
    g = GpuContext(scene, p)
    o = OracleScene(scene, p)
    K, spp = 24, 16
    tg, to = [], []
    for k in range(K):
        g.clear()
        g.render(spp, seed=100 + k)
        acc, light, _, splat = g.accumulators()
        tg.append(tile_means(combine(acc, light, spp, splat, g.npix), xres, yres))
        acc_o, light_o, splat_o = o.render(spp, seed=500 + k)
        to.append(tile_means(combine(acc_o, light_o, spp, splat_o, o.npix), xres, yres))
    tg, to = np.array(tg), np.array(to)
    se = np.sqrt(tg.var(0, ddof=1) / K + to.var(0, ddof=1) / K)
    z = np.abs(tg.mean(0) - to.mean(0)) / np.maximum(se, 1e-12)
    assert (z < 3.0).mean() >= 0.97, (z < 3.0).mean()
    assert np.all(z < 4.0), z.max()


@pytest.mark.parametrize("name", ["cornell_box", "cornell_box_medium"])
def test_pt2_matches_pt_in_bsdf_mode(gpu_lib, name):
    scene = getattr(scenes, name)(16, 16)
    means = []
    for algo, depth in ((abi.ALGO_PT, 8), (abi.ALGO_PT2, 9)):
        g = GpuContext(scene, make_params(max_ray_depth=depth, pt_sample_mode=abi.SAMPLE_BSDF, algo=algo))
        g.render(8192, seed=5)
        means.append(g.framebuffer().reshape(-1, 3).mean(axis=0))
    np.testing.assert_allclose(means[1], means[0], rtol=0.02)


def test_pt2_mis_matches_bsdf_with_one_light(gpu_lib):
    scene = scenes.cornell_box_medium(16, 16, one_light_triangle=True)
    means = []
    for mode in (abi.SAMPLE_BOTH, abi.SAMPLE_BSDF):
        g = GpuContext(scene, make_params(max_ray_depth=8, pt_sample_mode=mode, algo=abi.ALGO_PT2))
        g.render(8192, seed=9)
        means.append(g.framebuffer().reshape(-1, 3).mean(axis=0))
    np.testing.assert_allclose(means[0], means[1], rtol=0.02)


@pytest.mark.parametrize("qmc", [False, True])
def test_pt2_views_match_single_passes(gpu_lib, qmc):
    scene = scenes.cornell_box_medium(16, 16)
    params = make_params(max_ray_depth=8, wave_paths=500, algo=abi.ALGO_PT2, qmc=qmc)
    c = scene.camera
    views = [(c, 3), (copy.copy(c), 2)]
    views[1][0].xres, views[1][0].yres = 20, 12
    g = GpuContext(scene, params)
    imgs = g.render_views(views, seed=4)
    for v, ((cam, spp), img) in enumerate(zip(views, imgs)):
        s = copy.copy(scene)
        s.camera = cam
        one = GpuContext(s, make_params(max_ray_depth=8, algo=abi.ALGO_PT2, qmc=qmc))
        one.render(spp, 4 + v)
        ref = one.framebuffer().reshape(cam.yres, cam.xres, 3)
        np.testing.assert_allclose(img, ref, rtol=1e-4, atol=1e-5 * max(np.abs(ref).mean(), 1e-6))


def test_pt2_rejects_guiding_and_unknown_algo(gpu_lib):
    scene = scenes.cornell_box(8, 8)
    g = GpuContext(scene, make_params(max_ray_depth=6, algo=abi.ALGO_PT2))
    with pytest.raises(abi.TTError):
        g.set_guiding(True, 1)
    with pytest.raises(abi.TTError):
        GpuContext(scene, make_params(max_ray_depth=6, algo=7))


def test_pt2_rendering_algo(gpu_lib):
    from naivetrace_b200.algo import GpuPathTracer2
    algo = GpuPathTracer2(scenes.cornell_box(16, 16), make_params(max_ray_depth=8, max_spp=4))
    algo.run()
    assert algo.params.algo == abi.ALGO_PT2 and algo.params.max_ray_depth == 8
    acc, light, spp, _ = algo.ctx.accumulators()
    assert np.all(spp == 4) and np.all(light == 0)
    assert algo.generate_image().shape == (16, 16, 3)


@pytest.mark.parametrize("name", ["cornell_box_materials", "terrain_spheres_small", "cornell_box_media_mix"])
def test_pt2_qmc_per_path_parity(gpu_lib, name):
    """Quasi-random points (Sobol with per-pixel rotations) on both sides, over two passes so
    that the second pass's point indices continue after the first's."""
    scene = getattr(scenes, name)(32, 32) if name != "terrain_spheres_small" else scenes.terrain_spheres_small(48, 27)
    p = make_params(max_ray_depth=10, algo=abi.ALGO_PT2, qmc=True)
    g = GpuContext(scene, p)
    g.render(2, 3)
    g.render(2, 3)
    ag = g.accumulators()[0].reshape(-1, 3)
    o = OracleScene(scene, p)
    a0, _, _ = o.render(2, seed=3, sample_offset=0)
    a1, _, _ = o.render(2, seed=3, sample_offset=2)
    ao = (a0 + a1).reshape(-1, 3)
    assert g.stats()["error_flags"] == 0
    scale = max(np.abs(ao).mean(), 1e-6)
    close = np.all(np.abs(ag - ao) <= 1e-3 * np.abs(ao) + 1e-3 * scale, axis=1)
    assert close.mean() >= 0.93, close.mean()
    np.testing.assert_allclose(ag[close].sum(axis=0), ao[close].sum(axis=0), rtol=1e-3)


def test_pt2_qmc_lowers_error(gpu_lib):
    xres = yres = 32
    scene = scenes.cornell_box(xres, yres)
    ref = GpuContext(scene, make_params(max_ray_depth=3, algo=abi.ALGO_PT2))
    ref.render(16384, seed=77)
    R = ref.framebuffer().astype(np.float64)
    errs = {}
    for qmc in (False, True):
        e = []
        for k in range(3):
            g = GpuContext(scene, make_params(max_ray_depth=3, algo=abi.ALGO_PT2, qmc=qmc))
            g.render(64, seed=10 + k)
            I = g.framebuffer().astype(np.float64)
            e.append(np.mean((I - R) ** 2 / (R * R + 1e-2)))
        errs[qmc] = np.mean(e)
    assert errs[True] < 0.85 * errs[False], errs
    with pytest.raises(abi.TTError):
        GpuContext(scene, make_params(max_ray_depth=40, algo=abi.ALGO_PT2, qmc=True))
