"""Analytic spheres and the tabulated planetary atmosphere on the GPU against the oracle
(GPU): the batch intersector on sphere scenes (hit ids and distances, the reference's
known answer and its planet-radius self-intersection stress tests), and per-path and
tile parity of renders with spheres, a medium inside a glass sphere, an emissive sphere,
and an atmosphere seen from the ground (fisheye) and from space."""
import math

import numpy as np
import pytest

from naivetrace_b200 import abi, scenes
from naivetrace_b200.algo import GpuContext
from naivetrace_b200.scene import CameraSpec, Scene, diffuse, make_params
from oracle.oracle import OracleScene, combine
from test_gpu_render import render_both, tile_means
from test_oracle_spheres_atmosphere import hemisphere, offset_origin, surface_point

pytestmark = pytest.mark.gpu

LARGE = 3.4028234663852886e38 / 16


def sphere_scene(spheres, tris=False):
    s = Scene()
    m = s.add_material(diffuse(0.5))
    if tris:
        s.add_mesh(np.array([[-3, -3, 5], [3, -3, 5], [0, 3, 5]], float), np.array([[0, 1, 2]]), m)
    for c, r in spheres:
        s.add_sphere(c, r, m)
    s.camera = CameraSpec(xres=2, yres=2)
    return s


def test_sphere_batch_matches_oracle(gpu_lib):
    rng = np.random.default_rng(11)
    spheres = [(rng.uniform(-2, 2, 3), rng.uniform(0.1, 0.8)) for _ in range(40)]
    scene = sphere_scene(spheres, tris=True)
    g = GpuContext(scene, make_params())
    o = OracleScene(scene, make_params())
    n = 20000
    org = rng.uniform(-4, 4, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([org, np.zeros((n, 1)), d, np.full((n, 1), LARGE)], axis=1).astype(np.float32)
    pg, tg, _, _ = g.intersect(rays)
    po, to, _, _ = o.intersect(rays.astype(np.float64))
    assert (pg == po).mean() >= 0.9999
    hit = (pg == po) & (po >= 0)
    assert hit.sum() > n // 10
    np.testing.assert_allclose(tg[hit], to[hit], rtol=1e-5, atol=1e-6)


def test_sphere_known_answer_gpu(gpu_lib):
    g = GpuContext(sphere_scene([((0.0, 0.0, 2.0), 2.0)]), make_params())
    prim, t, _, _ = g.intersect(np.array([[0, 0, -1, 0, 0, 0, 1, LARGE]], np.float32))
    assert prim[0] == 0 and abs(t[0] - 1.0) < 1e-6


@pytest.mark.parametrize("case", ["outside", "inside", "shell"])
def test_sphere_self_intersection_gpu(gpu_lib, case):
    """The planet-radius stress tests, 64 independent chains stepped together."""
    R1, R2 = 6300.0, 6350.0
    c0 = np.array([0.0, 0.0, 2.0])
    spheres = {"outside": [(c0, R1)], "inside": [(c0, R1)], "shell": [(np.zeros(3), R1), (np.zeros(3), R2)]}[case]
    g = GpuContext(sphere_scene(spheres), make_params())
    rng = np.random.default_rng(5)
    chains = 64
    if case == "outside":
        for _ in range(100 // chains + 1):
            org = np.array([c0 + R1 * 10 * hemisphere(rng.normal(size=3), rng) for _ in range(chains)])
            tgt = np.array([c0 + R1 * 0.99 * rng.uniform() * hemisphere(np.array([0, 0, 1.0]), rng)
                            for _ in range(chains)])
            d = (tgt - org) / np.linalg.norm(tgt - org, axis=1, keepdims=True)
            prim, t, _, _ = g.intersect(np.concatenate([org, np.zeros((chains, 1)), d, np.full((chains, 1), LARGE)], 1)
                                        .astype(np.float32))
            assert np.all(prim == 0)
            rays = []
            for k in range(chains):
                pos, n = surface_point(c0, R1, org[k].astype(np.float32), d[k].astype(np.float32), float(t[k]))
                nd = hemisphere(n, rng)
                rays.append([*offset_origin(pos, n, nd), 0.0, *nd, LARGE])
            prim2, _, _, _ = g.intersect(np.array(rays, np.float32))
            assert np.all(prim2 == -1)
        return
    center = np.zeros(3) if case == "shell" else c0
    org = np.tile(np.array([0.5 * (R1 + R2), 0, 0]) if case == "shell" else c0, (chains, 1))
    d = np.tile(np.array([1.0, 0, 0]), (chains, 1))
    for _ in range(100):
        prim, t, _, _ = g.intersect(np.concatenate([org, np.zeros((chains, 1)), d, np.full((chains, 1), LARGE)], 1)
                                    .astype(np.float32))
        assert np.all(prim >= 0)
        for k in range(chains):
            cc, rr = spheres[prim[k]]
            pos, ng = surface_point(np.asarray(cc), rr, org[k].astype(np.float32).astype(np.float64),
                                    d[k].astype(np.float32).astype(np.float64), float(t[k]))
            rho = np.linalg.norm(pos - center)
            eps = R2 * np.finfo(np.float32).eps
            if case == "shell":
                assert R1 - eps <= rho <= R2 + eps
            n = ng if np.dot(ng, d[k]) < 0 else -ng
            d[k] = hemisphere(n, rng)
            org[k] = offset_origin(pos, ng, d[k])
            if case == "inside":
                assert np.linalg.norm(org[k] - c0) <= R1


SCENES = {
    "spheres_box": lambda r: scenes.spheres_box(r, r),
    "planet_atmosphere": lambda r: scenes.planet_atmosphere(r, r),
    "planet_from_space": lambda r: scenes.planet_from_space(r, r),
}


@pytest.mark.parametrize("name", list(SCENES))
def test_per_path_parity(gpu_lib, name):
    scene = SCENES[name](32)
    (ag, lg, sg), (ao, lo, so), g, o = render_both(scene, 4, 10)
    assert sg == so
    ag = ag.reshape(-1, 3)
    ao = ao.reshape(-1, 3)
    scale = max(np.abs(ao).mean(), 1e-6)
    close = np.all(np.abs(ag - ao) <= 1e-3 * np.abs(ao) + 1e-3 * scale, axis=1)
    assert close.mean() >= 0.9, close.mean()
    assert g.stats()["error_flags"] == 0


@pytest.mark.parametrize("name", list(SCENES))
def test_tile_z_test(gpu_lib, name):
    xres = yres = 64
    scene = SCENES[name](xres)
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
