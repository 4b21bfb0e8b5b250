"""End-to-end parity of the CUDA path tracer against the CPU oracle (GPU).

1. Per-path parity: both sides run the same PCG32 stream per camera sample, so at a few
   samples per pixel the accumulators agree pixel by pixel up to float rounding, except for
   the rare paths whose Russian-roulette or reflect/refract decision flips under it.
2. Statistical parity: 16x16 tile means of independent GPU and oracle renders agree within
   a 3-sigma z-test.
3. Convergence: relMSE against a converged render falls as 1/spp.
4. The RenderingAlgo-style host interface: schedule, callbacks, stop, image output.
"""
import threading

import numpy as np
import pytest

from naivetrace_b200 import abi, scenes
from naivetrace_b200.algo import GpuContext, GpuPathTracer
from naivetrace_b200.image import to_image
from naivetrace_b200.scene import make_params
from oracle.oracle import OracleScene, combine

pytestmark = pytest.mark.gpu


def render_both(scene, spp, depth, seed=1, mode=abi.SAMPLE_BOTH):
    p = make_params(max_ray_depth=depth, pt_sample_mode=mode)
    g = GpuContext(scene, p)
    g.render(spp, seed)
    acc_g, light_g, spp_g, splat_g = g.accumulators()
    o = OracleScene(scene, p)
    acc_o, light_o, splat_o = o.render(spp, seed=seed)
    return (acc_g, light_g, splat_g), (acc_o, light_o, splat_o), g, o


@pytest.mark.parametrize("name,depth", [("cornell_box", 10), ("cornell_box_materials", 10), ("terrain_spheres_small", 16)])
def test_per_path_parity(gpu_lib, name, depth):
    scene = getattr(scenes, name)(32, 32) if name != "terrain_spheres_small" else scenes.terrain_spheres_small(48, 27)
    (ag, lg, sg), (ao, lo, so), g, o = render_both(scene, 4, depth)
    assert sg == so
    ag = ag.reshape(-1, 3)
    ao = ao.reshape(-1, 3)
    scale = max(np.abs(ao).mean(), 1e-6)
    close = np.all(np.abs(ag - ao) <= 1e-3 * np.abs(ao) + 1e-3 * scale, axis=1)
    assert close.mean() >= 0.97, close.mean()
    # Over the pixels whose paths did not diverge the sums agree to float rounding.
    np.testing.assert_allclose(ag[close].sum(axis=0), ao[close].sum(axis=0), rtol=1e-4)
    # Camera-vertex splats (next-event estimation seen directly by the camera).
    np.testing.assert_allclose(lg.sum(), lo.sum(), rtol=0.02, atol=1e-6)


def test_peaked_env_map_per_path_parity(gpu_lib):
    """Env-map light samples invert the row and column CMFs through guide tables (a bisection
    only between the guide entries around the random number).  On a sky with bright spots
    (rows and columns where the CMFs jump by orders of magnitude, so that one guide interval
    spans many texels and many intervals none) the per-path results still match the oracle's
    full inversion."""
    from naivetrace_b200.scene import env_map
    scene = scenes.terrain_spheres_small(48, 27)
    tex = np.array(scene.env_lights[0].texture, dtype=np.float32).reshape(64, 128, 3).copy()
    tex *= 0.05
    tex[10:12, 40:43] = 400.0       # a small hot spot
    tex[20, 5:120] = 30.0           # a bright streak along one row
    tex[30:40, 90] = 60.0           # and down one column
    scene.env_lights[0] = env_map(tex, up=(0.0, 1.0, 0.0))
    (ag, lg, sg), (ao, lo, so), g, o = render_both(scene, 4, 16)
    assert sg == so
    ag = ag.reshape(-1, 3)
    ao = ao.reshape(-1, 3)
    scale = max(np.abs(ao).mean(), 1e-6)
    close = np.all(np.abs(ag - ao) <= 1e-3 * np.abs(ao) + 1e-3 * scale, axis=1)
    assert close.mean() >= 0.97, close.mean()
    np.testing.assert_allclose(ag[close].sum(axis=0), ao[close].sum(axis=0), rtol=1e-4)
    np.testing.assert_allclose(lg.sum(), lo.sum(), rtol=0.02, atol=1e-6)
    assert g.stats()["error_flags"] == 0


def tile_means(rgb, xres, yres, tile=16):
    a = rgb.reshape(yres, xres, 3)
    ty, tx = yres // tile, xres // tile
    return a[: ty * tile, : tx * tile].reshape(ty, tile, tx, tile, 3).mean(axis=(1, 3))


@pytest.mark.parametrize("name", ["cornell_box", "cornell_box_materials"])
def test_tile_z_test(gpu_lib, name):
    """16x16 tile means of the GPU render against the oracle's: z = difference over the
    standard error estimated from K independent renders per side.  With 48 tile-channels
    per case a 3-sigma bound is exceeded by chance now and then, so at least 97 % must lie
    within 3 sigma and all within 4 sigma (about the family-wise 5 % bound for 48 tests)."""
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


def test_relmse_falls_as_one_over_spp(gpu_lib):
    xres = yres = 48
    scene = scenes.cornell_box(xres, yres)
    p = make_params(max_ray_depth=10)
    ref = GpuContext(scene, p)
    ref.render(4096, seed=77)
    R = ref.framebuffer().astype(np.float64)
    errs = []
    spps = [4, 16, 64]
    for spp in spps:
        vals = []
        for k in range(4):
            g = GpuContext(scene, p)
            g.render(spp, seed=1000 + 10 * spp + k)
            I = g.framebuffer().astype(np.float64)
            vals.append(np.mean((I - R) ** 2 / (R * R + 1e-2)))
        errs.append(np.mean(vals))
    ratios = [errs[i] / errs[i + 1] for i in range(len(errs) - 1)]
    for r in ratios:
        assert 2.5 < r < 6.0, (errs, ratios)


def test_sample_modes_agree(gpu_lib):
    scene = scenes.cornell_box(16, 16)
    means = []
    for mode in (abi.SAMPLE_BOTH, abi.SAMPLE_BSDF, abi.SAMPLE_LIGHTS):
        g = GpuContext(scene, make_params(max_ray_depth=10, pt_sample_mode=mode))
        g.render(4096, seed=5)
        means.append(g.framebuffer().reshape(-1, 3).mean(axis=0))
    np.testing.assert_allclose(means[1], means[0], rtol=0.02)
    np.testing.assert_allclose(means[2], means[0], rtol=0.02)


def test_generate_image_matches_to_image(gpu_lib):
    scene = scenes.cornell_box(40, 24)
    g = GpuContext(scene, make_params(max_ray_depth=5))
    g.render(8, seed=3)
    rgb = g.framebuffer()
    np.testing.assert_array_equal(g.image(False), to_image(rgb, 40, 24, False))
    np.testing.assert_array_equal(g.image(True), to_image(rgb, 40, 24, True))


def test_range_pass_and_counts(gpu_lib):
    scene = scenes.cornell_box(16, 16)
    g = GpuContext(scene, make_params(max_ray_depth=5))
    g.render(2, seed=1, pixel_begin=0, pixel_end=100)
    acc, light, spp, splat = g.accumulators()
    assert np.all(spp[:100] == 2) and np.all(spp[100:] == 0)
    assert splat == 200
    assert np.all(acc.reshape(-1, 3)[100:] == 0)


def test_schedule_callbacks_and_stop(gpu_lib):
    scene = scenes.cornell_box(32, 32)
    algo = GpuPathTracer(scene, make_params(max_ray_depth=5, max_spp=15))
    seen = []
    algo.set_interrupt_callback(lambda complete: seen.append((complete, algo.generate_image().shape)))
    algo.run()
    # 1 + 2 + 4 + 8 = 15 samples per pixel in four complete passes
    assert [c for c, _ in seen] == [True] * 4
    _, _, spp, _ = algo.ctx.accumulators()
    assert np.all(spp == 15)
    # A full stop requested before Run returns from the first pass immediately.
    algo2 = GpuPathTracer(scene, make_params(max_ray_depth=5, max_spp=1 << 20))
    algo2.request_full_stop()
    algo2.run()
    assert algo2.last_status in (abi.TT_OK, abi.TT_ERR_INTERRUPTED)
    # Interrupt from another thread produces an extra, incomplete-pass callback.
    algo3 = GpuPathTracer(scene, make_params(max_ray_depth=5, max_spp=7))
    flags = []

    def cb(complete):
        flags.append(complete)

    algo3.set_interrupt_callback(cb)
    t = threading.Thread(target=algo3.request_interrupt)
    t.start()
    t.join()
    algo3.run()
    assert False in flags and flags.count(True) == 3


def test_no_device_errors(gpu_lib):
    scene = scenes.terrain_spheres_small(64, 36)
    g = GpuContext(scene, make_params(max_ray_depth=16))
    g.render(8, seed=2)
    st = g.stats()
    assert st["error_flags"] == 0
    assert st["extension_rays"] >= 64 * 36 * 8
    rgb = g.framebuffer()
    assert np.all(np.isfinite(rgb))


@pytest.mark.parametrize("width", [2, 8])
@pytest.mark.parametrize("name", ["cornell_box_materials", "terrain_spheres_small"])
def test_per_path_parity_wide_bvh(gpu_lib, monkeypatch, name, width):
    """The same per-path parity with the binary layout or the 8-wide compressed BVH as the
    traversal layout (the default is the 4-wide collapse of the device-built tree)."""
    monkeypatch.setenv("TT_BVH_WIDTH", str(width))
    scene = scenes.cornell_box_materials(32, 32) if name != "terrain_spheres_small" else scenes.terrain_spheres_small(48, 27)
    (ag, lg, sg), (ao, lo, so), g, o = render_both(scene, 4, 10)
    assert g.stats()["bvh_node_bytes"] == {2: 64, 8: 80}[width]
    ag = ag.reshape(-1, 3)
    ao = ao.reshape(-1, 3)
    scale = max(np.abs(ao).mean(), 1e-6)
    close = np.all(np.abs(ag - ao) <= 1e-3 * np.abs(ao) + 1e-3 * scale, axis=1)
    assert close.mean() >= 0.97, close.mean()


@pytest.mark.parametrize("name", ["cornell_box_materials", "terrain_spheres_small", "cornell_box_media_mix"])
def test_material_sorted_shading(gpu_lib, name):
    """Shading in material-sorted order (tt_params.sort_shading) changes which thread
    shades which path, not what a path computes: the same accumulators as the unsorted
    pass up to the order of the float atomics, and per-path parity with the oracle."""
    scene = getattr(scenes, name)(48, 32) if name != "terrain_spheres_small" else scenes.terrain_spheres_small(48, 27)
    depth = 12
    g0 = GpuContext(scene, make_params(max_ray_depth=depth, sort_shading=False))
    g0.render(4, seed=3)
    a0, l0, _, _ = g0.accumulators()
    g1 = GpuContext(scene, make_params(max_ray_depth=depth, sort_shading=True))
    g1.render(4, seed=3)
    a1, l1, _, _ = g1.accumulators()
    assert g1.stats()["error_flags"] == 0
    np.testing.assert_allclose(a1, a0, rtol=1e-4, atol=1e-6 * max(np.abs(a0).max(), 1e-9))
    np.testing.assert_allclose(l1, l0, rtol=1e-4, atol=1e-6 * max(np.abs(l0).max(), 1e-9))
    o = OracleScene(scene, make_params(max_ray_depth=depth))
    ao, lo, so = o.render(4, seed=3)
    ag, ao = a1.reshape(-1, 3), ao.reshape(-1, 3)
    scale = max(np.abs(ao).mean(), 1e-6)
    close = np.all(np.abs(ag - ao) <= 1e-3 * np.abs(ao) + 1e-3 * scale, axis=1)
    assert close.mean() >= 0.9, close.mean()
