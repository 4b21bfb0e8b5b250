"""The cube-map chi-square harness applied to the oracle's own shader samples (CPU): pins
the harness and the oracle's SampleBSDF/EvaluateBSDF consistency before the device
samples are judged by it."""
import numpy as np
import pytest

from naivetrace_b200.scene import CameraSpec, Scene, make_params
from oracle.oracle import OracleScene
from test_gpu_bsdf import LAMBDA, MATERIALS, chi2_pvalue, cube_bin, cube_cell_quadrature, incident


@pytest.fixture(scope="module")
def oracle_scene(oracle_lib):
    s = Scene()
    ids = {k: s.add_material(m) for k, m in MATERIALS.items()}
    s.add_mesh(np.array([[-1, -1, 0], [1, -1, 0], [0, 1, 0]], float), np.array([[0, 1, 2]]), ids["lambert"])
    s.camera = CameraSpec(xres=2, yres=2)
    return OracleScene(s, make_params()), ids


@pytest.mark.parametrize("mat", ["lambert", "beckmann_04", "beckmann_01"])
@pytest.mark.parametrize("inc", ["VERTICAL", "EXACT_45DEG", "ALMOST_45DEG", "MUCH_DEFLECTED"])
def test_chi_square_oracle_samples(oracle_scene, mat, inc):
    o, ids = oracle_scene
    wi = incident(inc)
    dirs, _, pdf = o.sample_bsdf(ids[mat], wi, LAMBDA, 50000, seed=777)
    ok = np.isfinite(dirs).all(axis=1) & (pdf > 0)
    counts = np.bincount(cube_bin(dirs[ok]), minlength=96)
    qd, qw = cube_cell_quadrature()
    _, qp = o.eval_bsdf(ids[mat], wi, LAMBDA, qd)
    ep = np.bincount(cube_bin(qd), weights=qp * qw, minlength=96)
    assert abs(ep.sum() - 1) < 2e-3
    assert chi2_pvalue(counts, ep / ep.sum() * ok.sum()) >= 0.01


@pytest.mark.parametrize("side", [1.0, -1.0])
@pytest.mark.parametrize("inc", ["VERTICAL", "EXACT_45DEG", "ALMOST_45DEG"])
def test_glossy_dielectric_oracle(oracle_scene, side, inc):
    """GlossyTransmissiveDielectricShader (IOR 1.3, alpha 0.2), lit from either side: the
    oracle's samples pass the chi-square against its own pdf, and the Monte Carlo scattered
    fraction E[f |cos| / pdf] agrees with the cubature integral of f |cos|, which is near 1
    (the reference's Albedo(1) for these cases, tests_sampling.cxx:1584-1606)."""
    o, ids = oracle_scene
    wi = side * incident(inc)
    n = 60000
    dirs, val, pdf = o.sample_bsdf(ids["glossy_glass"], wi, LAMBDA, n, seed=321)
    ok = np.isfinite(dirs).all(axis=1) & (pdf > 0)
    counts = np.bincount(cube_bin(dirs[ok]), minlength=96)
    qd, qw = cube_cell_quadrature()
    qv, qp = o.eval_bsdf(ids["glossy_glass"], wi, LAMBDA, qd)
    ep = np.bincount(cube_bin(qd), weights=qp * qw, minlength=96)
    assert abs(ep.sum() - 1) < 5e-3
    assert chi2_pvalue(counts, ep / ep.sum() * ok.sum()) >= 0.01
    w = np.where(ok, val[:, 0] * np.abs(dirs[:, 2]) / np.where(ok, pdf, 1.0), 0.0)
    integral = float((qv[:, 0] * np.abs(qd[:, 2]) * qw).sum())
    assert abs(w.mean() - integral) < 4 * w.std() / np.sqrt(n) + 3e-3
    assert abs(integral - 1.0) < 0.02
