"""Participating media in the oracle (CPU): the medium tracker's sequence of media along a
ray (MediaTransmission1/2, tests3.cxx:70-152), transmittance and volume pdf coefficients
through two boxes of homogeneous medium (TransmittanceEstimate, tests3.cxx:230-268),
spectral tracking to the next interaction (NextInteractionEstimation, tests3.cxx:271-344)
and the phase functions' sampling consistency (tests_sampling.cxx:1202-1233)."""
import math

import numpy as np
import pytest

from naivetrace_b200 import abi, scenes
from naivetrace_b200.scene import CameraSpec, MediumSpec, Scene, make_params, volume_boundary
from oracle.oracle import OracleScene, phase_sample
from test_gpu_bsdf import chi2_pvalue, cube_bin, cube_cell_quadrature

LAMBDA = np.array([30, 18, 6], np.int32)  # bins near the red, green and blue primaries


def _scene_with_media(objects, media):
    """objects: [(vertices, triangles, medium index)]; media: [MediumSpec]."""
    s = Scene()
    mids = [s.add_medium(m) for m in media]
    mats = [s.add_material(volume_boundary(m)) for m in mids]
    for v, t, m in objects:
        s.add_mesh(v, t, mats[m])
    s.camera = CameraSpec(xres=2, yres=2)
    return OracleScene(s, make_params())


def _sphere(center, radius, level=4):
    v, t = scenes.icosphere(level)
    return v * radius + np.asarray(center, float), t


def _flat_medium(sigma_s, sigma_a, priority):
    return MediumSpec(sigma_s=np.full(36, float(sigma_s)), sigma_a=np.full(36, float(sigma_a)), priority=priority)


def test_media_transmission_spheres(oracle_lib):
    """Five overlapping spheres of two media along the z axis; the higher-priority medium
    wins where they overlap (MediaTransmission1)."""
    med = [_flat_medium(1, 2, 1), _flat_medium(1, 2, 2)]
    objs = [(*_sphere((0, 0, -1), 1), 0), (*_sphere((0, 0, 2), 1), 1), (*_sphere((0, 0, 3), 1), 0),
            (*_sphere((0, 0, 6), 1), 0), (*_sphere((0, 0, 6), 0.5), 1)]
    o = _scene_with_media(objs, med)
    # Slightly off the axis so that the ray meets no tessellation vertex.
    init, walk = o.medium_walk((1e-3, 2e-3, -10.0), (0, 0, 1))
    assert init == -1
    z = np.array([t for t, _ in walk]) - 10.0
    media = [m for _, m in walk]
    np.testing.assert_allclose(z, [-2, 0, 1, 2, 3, 4, 5, 5.5, 6.5, 7], atol=2e-3)
    assert media == [0, -1, 1, 1, 0, -1, 0, 1, 0, -1]


def test_media_transmission_boxes_from_inside(oracle_lib):
    """Three 2x2x2 boxes; the ray starts inside the first one and passes through the
    shared diagonal edge of each face, whose two triangles report the same crossing
    (MediaTransmission2)."""
    med = [_flat_medium(1, 2, 1), _flat_medium(1, 2, 2)]
    objs = [(*scenes.centered_box((0, 0, -1), 1), 0), (*scenes.centered_box((0, 0, 2), 1), 1),
            (*scenes.centered_box((0, 0, 3), 1), 0)]
    o = _scene_with_media(objs, med)
    init, walk = o.medium_walk((0, 0, -1.0), (0, 0, 1))
    assert init == 0
    np.testing.assert_allclose([t for t, _ in walk], [1, 2, 3, 4, 5], atol=1e-6)
    assert [m for _, m in walk] == [-1, 1, 1, 0, -1]


def _two_unit_boxes(sigma_s, sigma_a, phase=abi.PHASE_UNIFORM):
    med = MediumSpec(sigma_s=np.full(36, float(sigma_s)), sigma_a=np.full(36, float(sigma_a)), phase=phase)
    return _scene_with_media([(*scenes.centered_box((0, 0, 0), 0.5), 0), (*scenes.centered_box((0, 0, 2), 0.5), 0)],
                             [med])


def test_transmittance_estimate(oracle_lib):
    o = _two_unit_boxes(1.0, 2.0)
    T, (fwd, bwd, tr) = o.transmittance((0, 0, -10.0), (0, 0, 1), 20.0, LAMBDA)
    np.testing.assert_allclose(T, math.exp(-6.0), atol=1e-3)
    # The segment starts and ends in vacuum: zero scatter densities at both ends.
    assert abs(tr - math.exp(-6.0)) < 1e-6 and abs(fwd) < 1e-6 and abs(bwd) < 1e-6
    # Ending inside the second box: the forward coefficient carries its extinction.
    T, (fwd, bwd, tr) = o.transmittance((0, 0, -10.0), (0, 0, 1), 12.0 / 0.9999, LAMBDA)
    np.testing.assert_allclose(T, math.exp(-4.5), rtol=1e-9)
    assert abs(fwd - 3.0 * tr) < 1e-9 and bwd == 0.0


def test_next_interaction_estimation(oracle_lib):
    o = _two_unit_boxes(3.0, 0.0)
    n = 1000
    out = o.track((0, 0, -10.0), (0, 0, 1), LAMBDA, n, seed=5)
    interacted = out[:, 0] > 0
    w = out[:, 2:5]
    sig = out[:, 5:8]
    # Surfaces: none.  Every sample either scatters inside a box or escapes.
    x = out[interacted, 1] - 10.0
    assert ((x > -0.5) & (x < 0.5) | (x > 1.5) & (x < 2.5)).all()
    # Pdf coefficients at the interaction: transmittance of the path up to it, the
    # extinction there, and zero at the vacuum start (tests3.cxx:307-308).
    depth = np.where(x < 0.5, x + 0.5, 1.0 + (x - 1.5))
    tr = np.exp(-3.0 * depth)
    np.testing.assert_allclose(out[interacted, 10], tr, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(out[interacted, 8], 3.0 * tr, rtol=1e-9, atol=1e-12)
    assert (out[interacted, 9] == 0).all()
    escaped_mean = np.where(interacted[:, None], 0, w).sum(0) / n
    interacted_mean = np.where(interacted[:, None], w * sig, 0).sum(0) / n
    np.testing.assert_allclose(escaped_mean, math.exp(-6.0), atol=1e-2)
    np.testing.assert_allclose(interacted_mean, 1 - math.exp(-6.0), atol=1e-2)


def test_chromatic_tracking_is_unbiased(oracle_lib):
    """Spectral tracking with different extinction per wavelength: the escaped weights
    average to each wavelength's own transmittance."""
    s_sig = np.linspace(0.5, 2.0, 36)
    med = MediumSpec(sigma_s=s_sig, sigma_a=np.full(36, 0.1))
    o = _scene_with_media([(*scenes.centered_box((0, 0, 0), 0.5), 0)], [med])
    n = 40000
    out = o.track((0, 0, -10.0), (0, 0, 1), LAMBDA, n, seed=11)
    interacted = out[:, 0] > 0
    escaped_mean = np.where(interacted[:, None], 0, out[:, 2:5]).sum(0) / n
    expect = np.exp(-(s_sig[LAMBDA] + 0.1))
    # Per-sample weights are bounded by a few units here; 5 sigma of the sample mean.
    sd = np.where(interacted[:, None], 0, out[:, 2:5]).std(0) / math.sqrt(n)
    assert (np.abs(escaped_mean - expect) < 5 * sd + 1e-4).all()
    inter_mean = np.where(interacted[:, None], out[:, 2:5] * out[:, 5:8], 0).sum(0) / n
    albedo = s_sig[LAMBDA] / (s_sig[LAMBDA] + 0.1)
    sd = np.where(interacted[:, None], out[:, 2:5] * out[:, 5:8], 0).std(0) / math.sqrt(n)
    # Single-scatter albedo x probability of an interaction within the box.
    assert (np.abs(inter_mean - albedo * (1 - expect)) < 5 * sd + 1e-4).all()


# --- phase functions ----------------------------------------------------------------------
def phase_value(kind, g, mu):
    """Closed forms of the phase functions: uniform 1/(4 pi), Rayleigh 3/(16 pi)(1+mu^2),
    Henyey-Greenstein (1-g^2)/(4 pi (1+g^2-2 g mu)^1.5), mu = cosine of the scattering angle."""
    if kind == abi.PHASE_UNIFORM:
        return np.full_like(mu, 1 / (4 * math.pi))
    if kind == abi.PHASE_RAYLEIGH:
        return 3 / (16 * math.pi) * (1 + mu * mu)
    return (1 - g * g) / (4 * math.pi * (1 + g * g - 2 * g * mu) ** 1.5)


@pytest.mark.parametrize("kind,g", [(abi.PHASE_UNIFORM, 0.0), (abi.PHASE_RAYLEIGH, 0.0),
                                    (abi.PHASE_HENYEY_GREENSTEIN, 0.4), (abi.PHASE_HENYEY_GREENSTEIN, 0.7),
                                    (abi.PHASE_HENYEY_GREENSTEIN, -0.3), (abi.PHASE_HENYEY_GREENSTEIN, 1e-4)])
@pytest.mark.parametrize("wi", [(0, 0, 1), (0.6, 0.0, -0.8)])
def test_phase_sampling_chi_square(oracle_lib, kind, g, wi):
    wi = np.asarray(wi, float)
    n = 50000
    dirs, pdf, val = phase_sample(kind, g, wi, n, seed=3)
    mu = dirs @ -wi
    np.testing.assert_allclose(np.linalg.norm(dirs, axis=1), 1, atol=1e-12)
    np.testing.assert_allclose(pdf, val, rtol=1e-12)
    np.testing.assert_allclose(pdf, phase_value(kind, g, mu), rtol=1e-9)
    counts = np.bincount(cube_bin(dirs), minlength=96)
    qd, qw = cube_cell_quadrature()
    ep = np.bincount(cube_bin(qd), weights=phase_value(kind, g, qd @ -wi) * qw, minlength=96)
    assert abs(ep.sum() - 1) < 2e-3
    assert chi2_pvalue(counts, ep / ep.sum() * n) >= 0.01
