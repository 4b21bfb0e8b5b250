"""Device-drawn phase-function samples (GPU): the PhaseFunctionTests fixture of the
reference (tests_sampling.cxx:1202-1259) run on samples the device draws.

For each phase function the device draws samples through tt_sample_phase_batch:
- the same PCG32 stream per sample as the oracle's MediumPhaseSample, so directions,
  values and pdfs agree sample by sample up to float rounding;
- the value equals the pdf (a single phase function is its own density) and both equal the
  closed form at the sampled cosine;
- binned into the 96-cell cube map, the counts pass the chi-square test against the closed
  form integrated per cell (bins merged to >= 5 expected, p >= 0.01 per case; the reference
  uses p >= 0.05 for its five fixtures, the bound is tightened for the larger family here);
- no cell deviates from its expectation by more than 4 sigma (the reference's
  TestCountsDeviationFromSigma(3) on 5000 samples; with 200k samples over 96 cells and 14
  cases 4 sigma keeps the family-wise false alarm rate below 1 %);
- the pdf integrates to one over the sphere (CheckIntegral).
The atmosphere's SimpleCombined mixture (Rayleigh for molecules, Henyey-Greenstein for
aerosols, weighted by their sigma_s at the vertex altitude; phasefunctions.cxx:206-273) is
checked at several altitudes, where the mixture weights differ.
"""
import math

import numpy as np
import pytest

from naivetrace_b200 import abi, scenes
from naivetrace_b200.algo import GpuContext
from naivetrace_b200.scene import AtmosphereSpec, CameraSpec, MediumSpec, Scene, diffuse, make_params, volume_boundary
from oracle.oracle import OracleScene
from test_gpu_bsdf import chi2_pvalue, cube_bin, cube_cell_quadrature

pytestmark = pytest.mark.gpu

LAMBDA = np.array([23, 17, 9], np.int32)
N = 200000

HOMOGENEOUS = {
    "uniform": (abi.PHASE_UNIFORM, 0.0),
    "rayleigh": (abi.PHASE_RAYLEIGH, 0.0),
    "hg_0.4": (abi.PHASE_HENYEY_GREENSTEIN, 0.4),
    "hg_0.7": (abi.PHASE_HENYEY_GREENSTEIN, 0.7),
    "hg_0.76": (abi.PHASE_HENYEY_GREENSTEIN, 0.76),
    "hg_-0.3": (abi.PHASE_HENYEY_GREENSTEIN, -0.3),
    "hg_1e-4": (abi.PHASE_HENYEY_GREENSTEIN, 1e-4),
}
ATM_G = 0.76
ALTITUDES = [0.5, 3.0, 25.0]  # km above the surface: aerosol-, mixed- and molecule-dominated


def closed_form(kind, g, mu):
    if kind == abi.PHASE_UNIFORM:
        return np.full_like(mu, 1 / (4 * math.pi))
    if kind == abi.PHASE_RAYLEIGH:
        return 3 / (16 * math.pi) * (1 + mu * mu)
    return (1 - g * g) / (4 * math.pi * (1 + g * g - 2 * g * mu) ** 1.5)


@pytest.fixture(scope="module")
def homogeneous(gpu_lib):
    s = Scene()
    ids = {}
    for k, (kind, g) in HOMOGENEOUS.items():
        ids[k] = s.add_medium(MediumSpec(sigma_s=np.full(36, 1.0), sigma_a=np.full(36, 0.1), phase=kind, phase_g=g))
    m = s.add_material(diffuse(0.5))
    s.add_mesh(np.array([[-1, -1, 0], [1, -1, 0], [0, 1, 0]], float), np.array([[0, 1, 2]]), m)
    s.camera = CameraSpec(xres=2, yres=2)
    return GpuContext(s), OracleScene(s, make_params()), ids


@pytest.fixture(scope="module")
def atmosphere(gpu_lib):
    tab = scenes.earth_atmosphere_table()
    s = Scene()
    atm = AtmosphereSpec(planet_center=(0.0, 0.0, 0.0), planet_radius=6371.0, h0=-1.0, dh=0.5, sigma_t=tab[0],
                         sigma_s_molecules=tab[1], sigma_s_aerosols=tab[2], g=ATM_G)
    mid = s.add_medium(atm)
    s.add_sphere((0.0, 0.0, 0.0), 6371.0 + atm.top_altitude, s.add_material(volume_boundary(mid)))
    s.camera = CameraSpec(xres=2, yres=2)
    return GpuContext(s), OracleScene(s, make_params()), mid


def incident(name):
    v = {"up": (0.0, 0.0, 1.0), "oblique": (0.6, 0.0, -0.8), "skew": (0.3, -0.4, math.sqrt(0.75))}[name]
    return np.asarray(v, float)


def check_distribution(dirs, pdf_of_dirs):
    """Chi-square and per-cell deviation of device directions against a density."""
    counts = np.bincount(cube_bin(dirs.astype(np.float64)), minlength=96)
    qd, qw = cube_cell_quadrature()
    ep = np.bincount(cube_bin(qd), weights=pdf_of_dirs(qd) * qw, minlength=96)
    assert abs(ep.sum() - 1) < 2e-3, ep.sum()  # CheckIntegral
    expected = ep / ep.sum() * len(dirs)
    sigma = np.sqrt(expected * (1 - ep / ep.sum()))
    dev = np.abs(counts - expected) / np.maximum(sigma, 1e-12)
    assert dev[expected > 5].max() < 4.0, dev.max()
    p = chi2_pvalue(counts, expected)
    assert p >= 0.01, p


@pytest.mark.parametrize("name", list(HOMOGENEOUS))
@pytest.mark.parametrize("inc", ["up", "oblique"])
def test_homogeneous_phase_device_samples(homogeneous, name, inc):
    g_ctx, o, ids = homogeneous
    kind, g = HOMOGENEOUS[name]
    g32 = float(np.float32(g))
    wi = incident(inc)
    pos = np.zeros(3)
    dg, vg, pg = g_ctx.sample_phase(ids[name], pos, wi, LAMBDA, N, seed=12356)
    assert np.isfinite(dg).all() and (pg > 0).all()
    np.testing.assert_allclose(np.linalg.norm(dg, axis=1), 1, atol=2e-6)
    # value = pdf = closed form at the sampled cosine
    np.testing.assert_allclose(vg, np.repeat(pg[:, None], 3, 1), rtol=1e-6)
    mu = dg.astype(np.float64) @ -wi
    np.testing.assert_allclose(pg, closed_form(kind, g32, mu), rtol=2e-3, atol=1e-6)
    # sample-by-sample parity with the oracle on the same streams
    do, vo, po = o.medium_phase_sample(ids[name], pos, wi, LAMBDA, 20000, seed=12356)
    same = np.all(np.abs(dg[:20000] - do) < 2e-3, axis=1)
    assert same.mean() >= 0.999, same.mean()
    np.testing.assert_allclose(pg[:20000][same], po[same], rtol=2e-3, atol=1e-6)
    check_distribution(dg, lambda qd: closed_form(kind, g32, qd @ -wi))
    # evaluation hook agrees with the closed form
    rng = np.random.default_rng(5)
    d = rng.normal(size=(4000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    ve, pe = g_ctx.eval_phase(ids[name], pos, wi, LAMBDA, d)
    np.testing.assert_allclose(pe, closed_form(kind, g32, d @ -wi), rtol=2e-3, atol=1e-6)
    np.testing.assert_allclose(ve[:, 0], pe, rtol=1e-6)


@pytest.mark.parametrize("alt", ALTITUDES)
@pytest.mark.parametrize("inc", ["up", "skew"])
def test_atmosphere_combined_phase_device_samples(atmosphere, alt, inc):
    g_ctx, o, mid = atmosphere
    wi = incident(inc)
    pos = np.array([0.0, 6371.0 + alt, 0.0])
    dg, vg, pg = g_ctx.sample_phase(mid, pos, wi, LAMBDA, N, seed=4)
    q = o.atmosphere_query(mid, pos, (0, 0, 0), (1, 0, 0), 1.0, LAMBDA)
    w0, w1 = q["sigma_s_mol"], q["sigma_s_aer"]
    sel0 = w0.sum() / (w0.sum() + w1.sum())
    g = float(np.float32(ATM_G))

    def density(d):
        m = d @ -wi
        return sel0 * closed_form(abi.PHASE_RAYLEIGH, 0.0, m) + (1 - sel0) * closed_form(abi.PHASE_HENYEY_GREENSTEIN, g, m)

    mu = dg.astype(np.float64) @ -wi
    ray = closed_form(abi.PHASE_RAYLEIGH, 0.0, mu)
    hg = closed_form(abi.PHASE_HENYEY_GREENSTEIN, g, mu)
    np.testing.assert_allclose(pg, sel0 * ray + (1 - sel0) * hg, rtol=3e-3, atol=1e-6)
    np.testing.assert_allclose(vg, (w0 / (w0 + w1))[None, :] * ray[:, None] + (w1 / (w0 + w1))[None, :] * hg[:, None],
                               rtol=3e-3, atol=1e-6)
    do, vo, po = o.medium_phase_sample(mid, pos, wi, LAMBDA, 20000, seed=4)
    same = np.all(np.abs(dg[:20000] - do) < 2e-3, axis=1)
    assert same.mean() >= 0.999, same.mean()
    check_distribution(dg, density)
    ve, pe = g_ctx.eval_phase(mid, pos, wi, LAMBDA, dg[:4000])
    np.testing.assert_allclose(pe, pg[:4000], rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(ve, vg[:4000], rtol=1e-5, atol=1e-7)
