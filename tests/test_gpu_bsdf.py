"""Device BSDF sampling and evaluation against the oracle (GPU).

Sample-by-sample parity: the device and the oracle draw from the same PCG32 stream per
sample, so directions, values and pdfs must agree up to float rounding.  The
distribution test restates SamplingConsistencyTest (tests_sampling.cxx:540-769): device
samples are binned into a cube map of 4x4 cells per face (96 bins), expected counts come
from integrating the oracle's pdf over each cell, bins are merged to >= 5 expected and a
chi-square test must give p >= 0.01 (the reference's fixtures use 0.05 per test; with a
dozen fixed-seed cases here the per-test bound is tightened to keep the family-wise false
alarm rate near 10 %).  Incident directions follow the reference's
parameterised cases VERTICAL / EXACT_45DEG / ALMOST_45DEG / MUCH_DEFLECTED
(tests_sampling.cxx:1265-1269).
"""
import math

import numpy as np
import pytest
from scipy import stats

from naivetrace_b200 import abi
from naivetrace_b200.algo import GpuContext
from naivetrace_b200.scene import (CameraSpec, MaterialSpec, Scene, dense_dielectric, diffuse, glass, glossy_glass,
                                   make_params, microfacet, mirror)
from naivetrace_b200.spectral import rgb_to_spectrum
from oracle.oracle import OracleScene

pytestmark = pytest.mark.gpu

LAMBDA = np.array([23, 17, 9], np.int32)  # LambdaIdxClosestToRGBPrimaries (spectral.hxx:59-62)


def incident(name):
    if name == "VERTICAL":
        return np.array([0.0, 0.0, 1.0])
    if name == "EXACT_45DEG":
        return np.array([0.0, 1.0, 1.0]) / math.sqrt(2)
    if name == "ALMOST_45DEG":
        v = np.array([0.0, 1.1, 1.0])
        return v / np.linalg.norm(v)
    v = np.array([0.0, 10.0, 1.0])  # MUCH_DEFLECTED
    return v / np.linalg.norm(v)


MATERIALS = {
    "lambert": diffuse(0.5),
    "mirror": mirror(0.9),
    "glass": glass(1.3),
    "beckmann_04": microfacet(0.3, 0.4),
    "beckmann_01": microfacet(rgb_to_spectrum((0.9, 0.6, 0.3)), 0.1),
    "glossy_glass": glossy_glass(1.3, 0.2),
    "dense": dense_dielectric(0.3, rgb_to_spectrum((0.8, 0.5, 0.2))),
}


@pytest.fixture(scope="module")
def contexts(gpu_lib):
    s = Scene()
    ids = {}
    for k, m in MATERIALS.items():
        ids[k] = s.add_material(m)
    s.add_mesh(np.array([[-1, -1, 0], [1, -1, 0], [0, 1, 0]], float), np.array([[0, 1, 2]]), ids["lambert"])
    s.camera = CameraSpec(xres=2, yres=2)
    return GpuContext(s), OracleScene(s, make_params()), ids


@pytest.mark.parametrize("mat", list(MATERIALS))
@pytest.mark.parametrize("inc", ["VERTICAL", "EXACT_45DEG", "ALMOST_45DEG", "MUCH_DEFLECTED"])
def test_samples_match_oracle(contexts, mat, inc):
    g, o, ids = contexts
    wi = incident(inc)
    n = 20000
    dg, vg, pg = g.sample_bsdf(ids[mat], wi, LAMBDA, n, seed=17)
    do, vo, po = o.sample_bsdf(ids[mat], wi, LAMBDA, n, seed=17)
    same_dir = np.all(np.abs(dg - do) < 2e-3, axis=1)
    assert same_dir.mean() >= 0.998, same_dir.mean()
    k = same_dir
    np.testing.assert_array_equal(np.signbit(pg[k]), np.signbit(po[k]))
    if mat == "glossy_glass":
        # The transmitted half vector's Jacobian 1 / (eta wi.h + wo.h)^2 has a pole; near it
        # (grazing incidence) float and double evaluations part, so 1 % of the samples may
        # differ beyond float rounding.
        close = np.isclose(pg[k], po[k], rtol=2e-3, atol=1e-6) & np.all(np.isclose(vg[k], vo[k], rtol=2e-3, atol=1e-5),
                                                                         axis=1)
        assert close.mean() >= 0.99, close.mean()
        return
    np.testing.assert_allclose(pg[k], po[k], rtol=2e-3, atol=1e-6)
    np.testing.assert_allclose(vg[k], vo[k], rtol=2e-3, atol=1e-5)


@pytest.mark.parametrize("mat", ["lambert", "beckmann_04", "beckmann_01", "glossy_glass", "dense"])
@pytest.mark.parametrize("inc", ["VERTICAL", "EXACT_45DEG", "MUCH_DEFLECTED"])
def test_eval_matches_oracle(contexts, mat, inc):
    g, o, ids = contexts
    wi = incident(inc)
    rng = np.random.default_rng(3)
    d = rng.normal(size=(5000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    vg, pg = g.eval_bsdf(ids[mat], wi, LAMBDA, d)
    vo, po = o.eval_bsdf(ids[mat], wi, LAMBDA, d)
    if mat == "glossy_glass":  # float vs double near the transmitted Jacobian's pole
        close = np.isclose(pg, po, rtol=2e-3, atol=1e-5) & np.all(np.isclose(vg, vo, rtol=2e-3, atol=1e-5), axis=1)
        assert close.mean() >= 0.995, close.mean()
        return
    np.testing.assert_allclose(pg, po, rtol=2e-3, atol=1e-5)
    np.testing.assert_allclose(vg, vo, rtol=2e-3, atol=1e-5)


# --- cube-map chi-square -----------------------------------------------------------------
CELLS = 4


def cube_bin(d):
    """Bin index of unit directions in a cube map with CELLS x CELLS cells per face."""
    a = np.abs(d)
    face_axis = np.argmax(a, axis=1)
    sign = np.take_along_axis(d, face_axis[:, None], 1)[:, 0] > 0
    face = face_axis * 2 + sign.astype(int)
    m = np.take_along_axis(a, face_axis[:, None], 1)[:, 0]
    uv_axes = np.array([[1, 2], [0, 2], [0, 1]])[face_axis]
    u = np.take_along_axis(d, uv_axes[:, :1], 1)[:, 0] / m
    v = np.take_along_axis(d, uv_axes[:, 1:], 1)[:, 0] / m
    iu = np.clip(((u + 1) * 0.5 * CELLS).astype(int), 0, CELLS - 1)
    iv = np.clip(((v + 1) * 0.5 * CELLS).astype(int), 0, CELLS - 1)
    return (face * CELLS + iu) * CELLS + iv


def cube_cell_quadrature(sub=128):
    """Directions and solid-angle weights of a midpoint rule over every cube cell."""
    g = (np.arange(CELLS * sub) + 0.5) / (CELLS * sub) * 2 - 1
    U, V = np.meshgrid(g, g, indexing="ij")
    U, V = U.ravel(), V.ravel()
    w = (2.0 / (CELLS * sub)) ** 2 / (1 + U * U + V * V) ** 1.5
    dirs, weights = [], []
    for axis in range(3):
        for s in (-1.0, 1.0):
            d = np.zeros((len(U), 3))
            ua, va = [[1, 2], [0, 2], [0, 1]][axis]
            d[:, axis] = s
            d[:, ua] = U
            d[:, va] = V
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            dirs.append(d)
            weights.append(w)
    return np.concatenate(dirs), np.concatenate(weights)


def chi2_pvalue(counts, expected):
    order = np.argsort(expected)
    c = counts[order].astype(float)
    e = expected[order].astype(float)
    # merge the smallest bins until every merged bin expects >= 5 (tests_stats.cxx:65-134)
    mc, me = [], []
    acc_c = acc_e = 0.0
    for ci, ei in zip(c, e):
        acc_c += ci
        acc_e += ei
        if acc_e >= 5:
            mc.append(acc_c)
            me.append(acc_e)
            acc_c = acc_e = 0.0
    if acc_e > 0 and me:
        mc[-1] += acc_c
        me[-1] += acc_e
    mc, me = np.array(mc), np.array(me)
    chi2 = np.sum((mc - me) ** 2 / me)
    dof = len(mc) - 1
    return 1.0 - stats.chi2.cdf(chi2, dof)


@pytest.mark.parametrize("mat", ["lambert", "beckmann_04", "beckmann_01"])
@pytest.mark.parametrize("inc", ["VERTICAL", "EXACT_45DEG", "ALMOST_45DEG", "MUCH_DEFLECTED"])
def test_chi_square_device_samples(contexts, mat, inc):
    g, o, ids = contexts
    wi = incident(inc)
    n = 100000
    dirs, _, pdf = g.sample_bsdf(ids[mat], wi, LAMBDA, n, seed=12356)
    ok = np.isfinite(dirs).all(axis=1) & (pdf > 0)
    counts = np.bincount(cube_bin(dirs[ok].astype(np.float64)), minlength=6 * CELLS * CELLS)
    qd, qw = cube_cell_quadrature()
    _, qp = o.eval_bsdf(ids[mat], wi, LAMBDA, qd)
    expected_prob = np.bincount(cube_bin(qd), weights=qp * qw, minlength=6 * CELLS * CELLS)
    total_prob = expected_prob.sum()
    assert abs(total_prob - 1.0) < 0.02, total_prob  # pdf normalised over the sphere
    p = chi2_pvalue(counts, expected_prob / total_prob * ok.sum())
    assert p >= 0.01, p


@pytest.mark.parametrize("inc", ["VERTICAL", "EXACT_45DEG", "MUCH_DEFLECTED"])
def test_lambert_albedo(contexts, inc):
    """Albedo of the Lambert 0.5 shader from device samples: E[f cos / pdf] = 0.5."""
    g, _, ids = contexts
    wi = incident(inc)
    d, v, pdf = g.sample_bsdf(ids["lambert"], wi, LAMBDA, 200000, seed=5)
    est = v[:, 0] * np.abs(d[:, 2]) / pdf
    assert abs(est.mean() - 0.5) < 1e-3


@pytest.mark.parametrize("inc", ["VERTICAL", "EXACT_45DEG", "ALMOST_45DEG"])
def test_glass_energy(contexts, inc):
    """Specular dielectric (IOR 1.3): reflect + transmit weights times |cos| / pmf sum to
    the Fresnel split; with the eta^2 radiance scaling undone the expectation is 1."""
    g, _, ids = contexts
    wi = incident(inc)
    d, v, pdf = g.sample_bsdf(ids["glass"], wi, LAMBDA, 100000, seed=9)
    w = v[:, 0] * np.abs(d[:, 2]) / np.abs(pdf)
    transmitted = d[:, 2] < 0
    w[transmitted] /= (1 / 1.3) ** 2
    assert abs(w.mean() - 1.0) < 5e-3


# --- glossy transmissive dielectric (GlossyTransmissiveDielectric cases, tests_sampling.cxx:1584-1620) ---
@pytest.mark.parametrize("side", [1.0, -1.0])
@pytest.mark.parametrize("inc", ["VERTICAL", "EXACT_45DEG", "ALMOST_45DEG", "MUCH_DEFLECTED"])
def test_glossy_dielectric_device_samples(contexts, side, inc):
    """IOR 1.3, alpha 0.2, lit from either side of the interface.  Device samples match the
    oracle's sample by sample; the Monte Carlo estimate of the scattered fraction
    E[f |cos| / pdf] equals the cubature integral of the oracle's f |cos| (CheckIntegral,
    near 1 for this lossless interface: the reference asserts albedo 1 except at grazing
    incidence); the sampled directions pass the cube-map chi-square against the oracle's pdf,
    except at grazing incidence where the reference disables the distribution test too."""
    g, o, ids = contexts
    wi = side * incident(inc)
    n = 200000
    dg, vg, pg = g.sample_bsdf(ids["glossy_glass"], wi, LAMBDA, n, seed=12356)
    do, vo, po = o.sample_bsdf(ids["glossy_glass"], wi, LAMBDA, 20000, seed=12356)
    same = np.all(np.abs(dg[:20000] - do) < 2e-3, axis=1)
    assert same.mean() >= 0.998, same.mean()
    close = np.isclose(pg[:20000][same], po[same], rtol=5e-3, atol=1e-5) & np.all(
        np.isclose(vg[:20000][same], vo[same], rtol=5e-3, atol=1e-5), axis=1)
    assert close.mean() >= 0.99, close.mean()  # float vs double near the Jacobian's pole
    ok = np.isfinite(dg).all(axis=1) & (pg > 0)
    w = np.where(ok, vg[:, 0].astype(np.float64) * np.abs(dg[:, 2]) / np.where(ok, pg, 1.0), 0.0)
    qd, qw = cube_cell_quadrature(256)
    qv, qp = o.eval_bsdf(ids["glossy_glass"], wi, LAMBDA, qd)
    integral = float((qv[:, 0] * np.abs(qd[:, 2]) * qw).sum())
    se = w.std() / math.sqrt(n)
    assert abs(w.mean() - integral) < 4 * se + 2e-3, (w.mean(), integral, se)
    if inc != "MUCH_DEFLECTED":
        assert abs(integral - 1.0) < 0.02, integral
        counts = np.bincount(cube_bin(dg[ok].astype(np.float64)), minlength=6 * CELLS * CELLS)
        ep = np.bincount(cube_bin(qd), weights=qp * qw, minlength=6 * CELLS * CELLS)
        assert abs(ep.sum() - 1.0) < 0.01, ep.sum()
        assert chi2_pvalue(counts, ep / ep.sum() * ok.sum()) >= 0.01
