"""The CPU oracle of the null-path tracer (--algo pt2) against the plain tracer and
against itself in its other sampling modes.

1. BSDF sampling only: pt2 with max_ray_depth D + 1 collects emission at the same path
   vertices as pt with D (pt2's node count starts at 2 and has no Russian roulette), so the
   two estimate the same image; also in a medium, where pt2's hero-wavelength delta
   tracking replaces pt's spectral tracking.
2. With exactly one light the MIS combination of light and BSDF sampling estimates the
   same image as BSDF sampling alone, with and without a medium.  (With more than one light
   the reference's light-sample pdf leaves out the selection probability, so its MIS weights
   do not sum to one; the oracle keeps that.)
3. Basic properties: finite accumulators with a positive mean (single pixels may go
   negative: RGB of a three-wavelength selection); no camera-vertex splats.

Image means of K independent renders per side are compared with a z-test at 4 sigma.
"""
import numpy as np
import pytest

from naivetrace_b200 import abi, scenes
from naivetrace_b200.scene import make_params
from oracle.oracle import OracleScene, combine


def _means(scene, params, K, spp, seed0):
    o = OracleScene(scene, params)
    out = []
    for k in range(K):
        acc, light, splat = o.render(spp, seed=seed0 + k)
        out.append(combine(acc, light, spp, splat, o.npix).reshape(-1, 3).mean(axis=0))
    return np.array(out)


def _agree(a, b, zmax=4.0):
    se = np.sqrt(a.var(0, ddof=1) / len(a) + b.var(0, ddof=1) / len(b))
    z = np.abs(a.mean(0) - b.mean(0)) / np.maximum(se, 1e-12)
    assert np.all(z < zmax), (a.mean(0), b.mean(0), z)


@pytest.mark.parametrize("name", ["cornell_box", "cornell_box_medium"])
def test_pt2_bsdf_mode_matches_pt(name):
    scene = getattr(scenes, name)(12, 12)
    d = 8
    a = _means(scene, make_params(max_ray_depth=d, pt_sample_mode=abi.SAMPLE_BSDF), 12, 64, 10)
    b = _means(scene, make_params(max_ray_depth=d + 1, pt_sample_mode=abi.SAMPLE_BSDF, algo=abi.ALGO_PT2), 12, 64, 50)
    _agree(a, b)


@pytest.mark.parametrize("name", ["cornell_box", "cornell_box_medium"])
def test_pt2_mis_matches_bsdf_with_one_light(name):
    scene = getattr(scenes, name)(12, 12, one_light_triangle=True)
    p_mis = make_params(max_ray_depth=8, algo=abi.ALGO_PT2)
    p_bsdf = make_params(max_ray_depth=8, pt_sample_mode=abi.SAMPLE_BSDF, algo=abi.ALGO_PT2)
    a = _means(scene, p_mis, 12, 32, 100)
    b = _means(scene, p_bsdf, 12, 64, 200)
    _agree(a, b)
    # MIS lowers the variance against BSDF sampling alone at equal sample count.
    a2 = _means(scene, p_mis, 6, 64, 300)
    assert a2.std(0).mean() < b.std(0).mean()


def test_pt2_accumulators():
    scene = scenes.cornell_box_materials(16, 16)
    o = OracleScene(scene, make_params(max_ray_depth=10, algo=abi.ALGO_PT2))
    acc, light, splat = o.render(4, seed=3)
    assert np.all(np.isfinite(acc)) and acc.mean() > 0
    assert np.all(light == 0)          # no next-event estimation at the camera
