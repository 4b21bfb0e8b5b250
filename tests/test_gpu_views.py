"""Multi-view batches (tt_render_views) against single-camera passes (GPU).

A batch renders every view in one wavefront, its later waves replayed from one captured
CUDA graph.  View v draws the random streams of a single-camera pass of that camera with
seed + v, so each view's image must equal the single-camera render pixel for pixel (up to
the order of float atomics): checked with one wave, with many graph-replayed waves, with
media (per-view medium trackers) and with fisheye and pinhole cameras mixed.
"""
import copy

import numpy as np
import pytest

from naivetrace_b200 import abi, scenes
from naivetrace_b200.algo import GpuContext
from naivetrace_b200.scene import CameraSpec, make_params

pytestmark = pytest.mark.gpu


def _views(scene):
    c = scene.camera
    return [
        (CameraSpec(kind=abi.CAMERA_PINHOLE, pos=c.pos, dir=c.dir, up=c.up, fov_deg=c.fov_deg, xres=24, yres=16), 4),
        (CameraSpec(kind=abi.CAMERA_PINHOLE, pos=(0.2, 0.6, -0.8), dir=(0.3, -0.1, 1.0), up=(0, 1, 0), fov_deg=55.0,
                    xres=17, yres=23), 2),
        (CameraSpec(kind=abi.CAMERA_PINHOLE, pos=(0.5, 0.5, -1.4), dir=(0, 0, 1), up=(0, 1, 0), fov_deg=30.0,
                    xres=40, yres=40), 3),
        (CameraSpec(kind=abi.CAMERA_FISHEYE, pos=(0.5, 0.5, 0.5), dir=(0, 1, 0), up=(0, 0, 1), fov_deg=90.0,
                    xres=20, yres=20), 2),
    ]


def _single(scene, cam, spp, seed, params):
    s = copy.copy(scene)
    s.camera = cam
    g = GpuContext(s, params)
    g.render(spp, seed)
    return g.framebuffer().reshape(cam.yres, cam.xres, 3).astype(np.float64)


@pytest.mark.parametrize("name,wave", [("cornell_box", 0), ("cornell_box", 600), ("cornell_box_medium", 500),
                                       ("cornell_box_materials", 0)])
def test_views_match_single_camera_passes(gpu_lib, name, wave):
    """wave = 600 paths per wave gives 6 waves: one eager, five replayed from the graph."""
    scene = getattr(scenes, name)(16, 16)
    params = make_params(max_ray_depth=8, wave_paths=wave)
    views = _views(scene)
    g = GpuContext(scene, params)
    imgs = g.render_views(views, seed=11)
    assert g.stats()["error_flags"] == 0
    for v, ((cam, spp), img) in enumerate(zip(views, imgs)):
        ref = _single(scene, cam, spp, 11 + v, make_params(max_ray_depth=8))
        scale = max(np.abs(ref).mean(), 1e-6)
        np.testing.assert_allclose(img, ref, rtol=1e-4, atol=1e-5 * scale, err_msg=f"view {v}")


def test_views_repeat_and_large_batch(gpu_lib):
    """Two calls give the same images (the batch state starts from zero every call); a
    batch of 40 views of uneven size renders without errors."""
    scene = scenes.terrain_spheres_small(32, 18)
    g = GpuContext(scene, make_params(max_ray_depth=6, wave_paths=20000))
    views = [(c if c.xres <= 128 else CameraSpec(kind=c.kind, pos=c.pos, dir=c.dir, up=c.up, fov_deg=c.fov_deg,
                                                  xres=48, yres=48), 2)
             for c, _ in scenes.terrain_views(40, seed=3, resolutions=(16, 32, 64))]
    a = g.render_views(views, seed=5)
    b = g.render_views(views, seed=5)
    for x, y in zip(a, b):
        np.testing.assert_allclose(x, y, rtol=1e-5, atol=1e-6)
    assert all(np.isfinite(x).all() for x in a)
    assert sum(float(x.mean()) > 0 for x in a) >= 30
    assert g.stats()["error_flags"] == 0


def test_autotune_views(gpu_lib):
    scene = scenes.terrain_spheres_small(32, 18)
    g = GpuContext(scene, make_params(max_ray_depth=6))
    views = [(c, 2) for c, _ in scenes.terrain_views(8, seed=1, resolutions=(64, 128))]
    r = g.autotune_views(views)
    assert r["wave_paths"] in (1 << 22, 1 << 24, 1 << 25, 1 << 26)
    assert r["grid"] > 0 and r["ms"] > 0
    # 12 queue-capacity x launch-width probes, then half-size blocks and the 8-wide BVH.
    assert len(r["candidates"]) == 14
    assert {c["block"] for c in r["candidates"]} == {128, 256}
    assert {c["bvh_width"] for c in r["candidates"]} == {4, 8}  # the device-built default, then 8-wide
    assert r["block"] in (128, 256) and r["bvh_width"] in (4, 8)
    assert r["ms"] == min(c["ms"] for c in r["candidates"])
    imgs = g.render_views(views, seed=2)
    assert len(imgs) == 8 and all(np.isfinite(i).all() for i in imgs)
    assert g.stats()["error_flags"] == 0
    # Whichever configuration won, the images are those of single-camera passes.
    for v in (0, 5):
        cam, spp = views[v]
        ref = _single(scene, cam, spp, 2 + v, make_params(max_ray_depth=6))
        scale = max(np.abs(ref).mean(), 1e-6)
        np.testing.assert_allclose(imgs[v].astype(np.float64), ref, rtol=1e-3, atol=1e-4 * scale)


def test_views_reject_bad_input(gpu_lib):
    scene = scenes.cornell_box(8, 8)
    g = GpuContext(scene, make_params(max_ray_depth=4))
    bad = [(CameraSpec(kind=abi.CAMERA_PINHOLE, xres=0, yres=8), 1)]
    with pytest.raises(abi.TTError):
        g.render_views(bad)
    with pytest.raises(abi.TTError):
        g.render_views([(scene.camera, 0)])


def test_views_per_path_against_oracle(gpu_lib):
    """A three-view batch against the CPU oracle per path: view v of the batch draws the
    streams of a single-camera pass with seed + v, which the oracle reproduces."""
    from oracle.oracle import OracleScene, combine
    scene = scenes.cornell_box_materials(16, 16)
    views = _views(scene)[:3]
    g = GpuContext(scene, make_params(max_ray_depth=8))
    imgs = g.render_views(views, seed=21)
    assert g.stats()["error_flags"] == 0
    for v, ((cam, spp), img) in enumerate(zip(views, imgs)):
        s = copy.copy(scene)
        s.camera = cam
        o = OracleScene(s, make_params(max_ray_depth=8))
        acc, light, splat = o.render(spp, seed=21 + v)
        ref = combine(acc, light, spp, splat, o.npix).reshape(cam.yres, cam.xres, 3)
        a, b = img.reshape(-1, 3).astype(np.float64), ref.reshape(-1, 3)
        scale = max(np.abs(b).mean(), 1e-6)
        close = np.all(np.abs(a - b) <= 2e-3 * np.abs(b) + 2e-3 * scale, axis=1)
        assert close.mean() >= 0.9, (v, close.mean())


def test_views_completion_times_and_guiding(gpu_lib):
    """Per-view completion times: within the batch's duration, ordered by the wave that
    finishes each view; a guided batch (learned guiding on) renders finite images."""
    scene = scenes.terrain_spheres_small(32, 18)
    g = GpuContext(scene, make_params(max_ray_depth=6, wave_paths=4000))
    views = [(c, 2) for c, _ in scenes.terrain_views(6, seed=2, resolutions=(32, 48))]
    g.render_views(views, seed=3)
    t = g.views_completion_ms(len(views))
    assert np.all(t > 0) and np.all(np.diff(t) >= -1e-3)  # later views finish in later waves
    g.set_guiding(True, 1, seed=7)
    for k in range(2):
        g.render_views([(c, 1) for c, _ in views], seed=10 + k)
    g.set_guiding(True, 0, seed=7)
    imgs = g.render_views(views, seed=4)
    assert all(np.isfinite(i).all() for i in imgs)
    assert g.stats()["guide_steps"] > 0 and g.stats()["error_flags"] == 0
