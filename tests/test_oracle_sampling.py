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
