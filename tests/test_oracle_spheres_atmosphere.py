"""Analytic spheres and the tabulated planetary atmosphere in the oracle (CPU).

Spheres: the reference's intersector known answer (IntersectorTests.Sphere,
tests.cxx:375-386) and its self-intersection stress tests at planetary radius
(SphereIntersectionMadness 1-3, tests.cxx:456-569), which bounce rays off a sphere of
radius 6300 with the anti-self-intersection offset and require that they neither re-hit
the surface they leave nor escape a closed sphere or shell.

Atmosphere: SphereGeometry's altitude and lowest point (SimpleAtmosphereTest,
tests.cxx:798-853), the collision coefficients of the exponential model tabulated, the
spectral tracking and ratio tracking estimators against the analytic transmittance of the
table, and the SimpleCombined phase function's sampling consistency.
"""
import math

import numpy as np
import pytest

from naivetrace_b200 import abi, scenes
from naivetrace_b200.scene import AtmosphereSpec, CameraSpec, Scene, diffuse, make_params, volume_boundary
from oracle.oracle import OracleScene
from test_gpu_bsdf import chi2_pvalue, cube_bin, cube_cell_quadrature

RGB_PRIMARY_BINS = np.array([23, 17, 9], np.int32)  # LambdaIdxClosestToRGBPrimaries, spectral.hxx:61-64
GAMMA5 = 5 * np.finfo(np.float32).eps / (1 - 5 * np.finfo(np.float32).eps)


def sphere_scene(spheres):
    s = Scene()
    m = s.add_material(diffuse(0.5))
    for c, r in spheres:
        s.add_sphere(c, r, m)
    s.camera = CameraSpec(xres=2, yres=2)
    return OracleScene(s, make_params())


def trace(o, org, d):
    prim, t, _, _ = o.intersect(np.array([[*org, 0.0, *d, 3.4e38 / 16]]))
    return int(prim[0]), float(t[0])


def surface_point(center, radius, org, d, t):
    n = np.asarray(org) + t * np.asarray(d) - center
    n = n / np.linalg.norm(n)
    return center + radius * n, n


def offset_origin(pos, n, d):
    """AntiSelfIntersectionOffset (scene.cxx:256-261) with FillPosBoundsSphere's bounds."""
    bounds = np.abs(pos.astype(np.float32).astype(np.float64)) * GAMMA5
    delta = np.dot(bounds, np.abs(n))
    return pos + delta * (1.0 if np.dot(d, n) > 0 else -1.0) * n


def hemisphere(n, rng):
    while True:
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        if np.dot(v, n) > 0:
            return v


def test_sphere_known_answer(oracle_lib):
    o = sphere_scene([((0.0, 0.0, 2.0), 2.0)])
    prim, t = trace(o, (0.0, 0.0, -1.0), (0.0, 0.0, 1.0))
    assert prim == 0 and abs(t - 1.0) < 1e-6
    pos, n = surface_point(np.array([0.0, 0.0, 2.0]), 2.0, (0, 0, -1), (0, 0, 1), t)
    np.testing.assert_allclose(pos, [0, 0, 0], atol=1e-6)
    np.testing.assert_allclose(n, [0, 0, -1], atol=1e-6)


def test_sphere_no_self_intersection_from_outside(oracle_lib):
    c, R = np.array([0.0, 0.0, 2.0]), 6300.0
    o = sphere_scene([(c, R)])
    rng = np.random.default_rng(3)
    for _ in range(100):
        org = c + R * 10 * hemisphere(rng.normal(size=3), rng)
        target = c + R * 0.99 * hemisphere(np.array([0, 0, 1.0]), rng) * rng.uniform()
        d = (target - org) / np.linalg.norm(target - org)
        prim, t = trace(o, org, d)
        assert prim == 0
        pos, n = surface_point(c, R, org, d, t)
        assert np.linalg.norm(org - pos) <= np.linalg.norm(org - c)
        nd = hemisphere(n, rng)
        prim2, _ = trace(o, offset_origin(pos, n, nd), nd)
        assert prim2 == -1


@pytest.mark.parametrize("shell", [False, True])
def test_sphere_bounces_stay_inside(oracle_lib, shell):
    """Bounce inside one sphere (radius 6300), or inside the shell between radii 6300 and
    6350: every hit lies on the spheres and no ray escapes."""
    R1, R2 = 6300.0, 6350.0
    c = np.zeros(3)
    spheres = [(c, R1), (c, R2)] if shell else [(np.array([0.0, 0.0, 2.0]), R1)]
    o = sphere_scene(spheres)
    rng = np.random.default_rng(7)
    org = np.array([0.5 * (R1 + R2), 0.0, 0.0]) if shell else np.array([0.0, 0.0, 2.0])
    d = np.array([1.0, 0.0, 0.0])
    for _ in range(100):
        prim, t = trace(o, org, d)
        assert prim >= 0
        cc, rr = spheres[prim]
        pos, ng = surface_point(np.asarray(cc), rr, org, d, t)
        rho = np.linalg.norm(pos - c)
        eps = R2 * np.finfo(np.float32).eps
        if shell:
            assert R1 - eps <= rho <= R2 + eps
        n = ng if np.dot(ng, d) < 0 else -ng  # oriented towards the incoming ray
        d = hemisphere(n, rng)
        org = offset_origin(pos, ng, d)
        if not shell:
            assert np.linalg.norm(org - np.array([0.0, 0.0, 2.0])) <= R1


# --- atmosphere ---------------------------------------------------------------------------
def atmosphere_scene(center=(0.0, 0.0, 0.0), radius=6371.0, table=None, h0=-1.0, dh=0.5, g=0.76):
    tab = scenes.earth_atmosphere_table(h0=h0, dh=dh) if table is None else table
    s = Scene()
    atm = AtmosphereSpec(planet_center=center, planet_radius=radius, h0=h0, dh=dh, sigma_t=tab[0],
                         sigma_s_molecules=tab[1], sigma_s_aerosols=tab[2], g=g)
    mid = s.add_medium(atm)
    s.add_sphere(center, radius + atm.top_altitude, s.add_material(volume_boundary(mid)))
    s.camera = CameraSpec(xres=2, yres=2)
    return OracleScene(s, make_params()), tab, atm


def test_altitude_and_lowest_point(oracle_lib):
    o, _, _ = atmosphere_scene(center=(0.0, 0.0, 1.0), radius=100.0)
    q = o.atmosphere_query(0, (0.0, 110.0, 1.0), (0, 0, 0), (1, 0, 0), 1.0, RGB_PRIMARY_BINS)
    assert abs(q["altitude"] - 10.0) < 1e-6
    # Looking down through the layer, limited, and looking up (tests.cxx:823-851).
    q = o.atmosphere_query(0, (0, 0, 0), (-1000.0, 0.0, 101.0), (1, 0, 0), 2000.0, RGB_PRIMARY_BINS)
    np.testing.assert_allclose(q["lowest"], [0, 0, 101], atol=1e-8)
    q = o.atmosphere_query(0, (0, 0, 0), (-1000.0, 0.0, 101.0), (1, 0, 0), 20.0, RGB_PRIMARY_BINS)
    np.testing.assert_allclose(q["lowest"], [-980, 0, 101], atol=1e-8)
    up = np.array([1.0, 0.0, 10.0]) / np.linalg.norm([1.0, 0.0, 10.0])
    q = o.atmosphere_query(0, (0, 0, 0), (0.0, 0.0, 101.0), up, 5.0, RGB_PRIMARY_BINS)
    np.testing.assert_allclose(q["lowest"], [0, 0, 101], atol=1e-8)


def test_collision_coefficients_of_the_exponential_model(oracle_lib):
    """SimpleAtmosphereTest.CollisionCoefficients (tests.cxx:807-820) on the tabulated
    exponential model: sigma_s and sigma_a at 10 km in the red primary bin within 1 %."""
    tab = scenes.simple_atmosphere_table()
    o, _, _ = atmosphere_scene(table=tab, dh=0.05)
    q = o.atmosphere_query(0, (0.0, 6371.0 + 10.0, 0.0), (0, 0, 0), (1, 0, 0), 1.0, RGB_PRIMARY_BINS)
    exp_s = math.exp(-10 / 8.0) * 0.0076 + math.exp(-10 / 1.2) * 20e-3
    exp_a = math.exp(-10 / 8.0) * 0.0 + math.exp(-10 / 1.2) * 2.22e-3
    assert abs(q["sigma_s"][0] - exp_s) < 1e-2 * exp_s
    assert abs((q["sigma_t"] - q["sigma_s"])[0] - exp_a) < 1e-2 * exp_a


def test_table_interpolation_and_clamping(oracle_lib):
    o, tab, atm = atmosphere_scene()
    tab = [a.astype(np.float32).astype(np.float64) for a in tab]  # the ABI carries float tables
    li = RGB_PRIMARY_BINS
    for alt in [-0.7, 0.0, 0.26, 7.3, 24.9, 150.1]:
        q = o.atmosphere_query(0, (0.0, 6371.0 + alt, 0.0), (0, 0, 0), (1, 0, 0), 1.0, li)
        ri = (alt - atm.h0) / atm.dh
        i = int(ri)  # truncation toward zero, as the reference's (int) cast
        f = ri - i
        lerp = lambda a: (1 - f) * a[i, li] + f * a[i + 1, li]
        np.testing.assert_allclose(q["sigma_s_mol"], lerp(tab[1]), rtol=1e-9)
        np.testing.assert_allclose(q["sigma_s_aer"], lerp(tab[2]), rtol=1e-9)
        np.testing.assert_allclose(q["sigma_t"], lerp(tab[0]), rtol=1e-9)
        np.testing.assert_allclose(q["sigma_s"], lerp(tab[1]) + lerp(tab[2]), rtol=1e-9)
        maj = np.maximum.accumulate(tab[0].max(axis=1)[::-1])[::-1]
        assert abs(q["majorant"] - ((1 - f) * maj[i] + f * maj[i + 1])) <= 1e-12 * maj[0]
    # Above the table: nothing; below its first row: the first row.
    q = o.atmosphere_query(0, (0.0, 6371.0 + 500.0, 0.0), (0, 0, 0), (1, 0, 0), 1.0, li)
    assert np.all(q["sigma_t"] == 0) and q["majorant"] == 0
    q = o.atmosphere_query(0, (0.0, 6371.0 - 5.0, 0.0), (0, 0, 0), (1, 0, 0), 1.0, li)
    np.testing.assert_allclose(q["sigma_t"], tab[0][0, li], rtol=1e-12)


def optical_depth(tab, atm, org, d, length, li, steps=200000):
    t = (np.arange(steps) + 0.5) * (length / steps)
    p = np.asarray(org)[None, :] + t[:, None] * np.asarray(d)[None, :]
    alt = np.linalg.norm(p - np.asarray(atm.planet_center), axis=1) - atm.planet_radius
    ri = (alt - atm.h0) / atm.dh
    i = np.clip(np.trunc(ri).astype(int), 0, len(tab[0]) - 2)
    f = (ri - i)[:, None]
    sig = (1 - f) * tab[0][i][:, li] + f * tab[0][i + 1][:, li]
    sig[ri >= len(tab[0]) - 1] = 0
    return sig.sum(axis=0) * (length / steps)


@pytest.mark.parametrize("elevation_deg", [90.0, 20.0])
def test_tracking_estimators_match_the_table(oracle_lib, elevation_deg):
    """Spectral tracking (escaped weights) and ratio tracking (transmittance estimates)
    both average to exp(-optical depth) of the tabulated coefficients along a ray from
    2 m above the ground out of the atmosphere."""
    o, tab, atm = atmosphere_scene()
    li = RGB_PRIMARY_BINS
    e = math.radians(elevation_deg)
    org = np.array([0.0, 6371.002, 0.0])
    d = np.array([math.cos(e), math.sin(e), 0.0])
    # Distance to the top of the atmosphere.
    b = np.dot(org, d)
    r_top = 6371.0 + atm.top_altitude
    length = -b + math.sqrt(b * b - (np.dot(org, org) - r_top * r_top))
    T = np.exp(-optical_depth(tab, atm, org, d, length, li))
    n = 20000
    out = o.track(org, d, li, n, seed=9)
    w = np.where((out[:, 0] > 0)[:, None], 0.0, out[:, 2:5])
    sd = w.std(axis=0) / math.sqrt(n)
    assert np.all(np.abs(w.mean(axis=0) - T) < 5 * sd + 2e-3), (w.mean(axis=0), T)
    est = np.array([o.transmittance(org, d, 2 * length, li, seed=s)[0] for s in range(3000)])
    sd = est.std(axis=0) / math.sqrt(len(est))
    assert np.all(np.abs(est.mean(axis=0) - T) < 5 * sd + 2e-3), (est.mean(axis=0), T)


def test_combined_phase_function(oracle_lib):
    """SimpleCombined of Rayleigh (molecules) and Henyey-Greenstein (aerosols) weighted by
    the constituents' sigma_s at the vertex altitude: value, pdf and sampled distribution."""
    o, tab, atm = atmosphere_scene(g=0.76)
    li = RGB_PRIMARY_BINS
    pos = np.array([0.0, 6371.0 + 1.3, 0.0])
    wi = np.array([0.3, -0.4, np.sqrt(1 - 0.25)])
    n = 60000
    dirs, val, pdf = o.medium_phase_sample(0, pos, wi, li, n, seed=4)
    q = o.atmosphere_query(0, pos, (0, 0, 0), (1, 0, 0), 1.0, li)
    w0, w1 = q["sigma_s_mol"], q["sigma_s_aer"]
    sel0 = w0.sum() / (w0.sum() + w1.sum())
    mu = dirs @ -wi
    ray = 3 / (16 * math.pi) * (1 + mu * mu)
    g = float(np.float32(0.76))  # the ABI carries g as a float
    hg = (1 - g * g) / (4 * math.pi * (1 + g * g - 2 * g * mu) ** 1.5)
    np.testing.assert_allclose(pdf, sel0 * ray + (1 - sel0) * hg, rtol=1e-9)
    np.testing.assert_allclose(val, (w0 / (w0 + w1))[None, :] * ray[:, None] + (w1 / (w0 + w1))[None, :] * hg[:, None],
                               rtol=1e-9)
    counts = np.bincount(cube_bin(dirs), minlength=96)
    qd, qw = cube_cell_quadrature()
    qmu = qd @ -wi
    qp = sel0 * 3 / (16 * math.pi) * (1 + qmu * qmu) + (1 - sel0) * (1 - g * g) / (
        4 * math.pi * (1 + g * g - 2 * g * qmu) ** 1.5)
    ep = np.bincount(cube_bin(qd), weights=qp * qw, minlength=96)
    assert abs(ep.sum() - 1) < 2e-3
    assert chi2_pvalue(counts, ep / ep.sum() * n) >= 0.01


def test_planet_scene_renders(oracle_lib):
    """The planet scene under a fisheye camera renders finite, positive sky radiance."""
    s = scenes.planet_atmosphere(16, 16)
    o = OracleScene(s, make_params(max_ray_depth=8))
    acc, light, splat = o.render(4, seed=1)
    img = acc.reshape(-1, 3) / 4
    assert np.all(np.isfinite(img)) and img.sum() > 0
