"""Seeded procedural scenes for the workloads the tracer is measured on.

- cornell_box():     unit-cube Cornell box with two boxes and a ceiling area light
                     (256x256, 16 spp, depth 10 as the standard small case).
- terrain_spheres(): 1024x1024-vertex fBm heightfield (~2.1 M triangles) with 32
                     tessellated spheres of 20 480 triangles each, lit by a float32
                     equirect sky gradient plus a 0.53 degree sun (1920x1080, 64 spp,
                     depth 16).
- small scenes for parity tests.
There is no public dataset involved; every input is generated here from a seed.
"""
from __future__ import annotations

import math

import numpy as np

from . import abi
from .scene import (AtmosphereSpec, CameraSpec, MediumSpec, Scene, area_light, dense_dielectric, diffuse, env_map, glass,
                    glossy_glass, microfacet, mirror, sun_light, volume_boundary)
from .spectral import band_spectrum, rgb_to_spectrum


def quad(p0, p1, p2, p3):
    """Two triangles (p0,p1,p2), (p0,p2,p3); winding normal = (p1-p0) x (p2-p0)."""
    v = np.array([p0, p1, p2, p3], dtype=np.float64)
    t = np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32)
    return v, t


def box_mesh(size, center_base, rot_y_deg):
    """Closed axis-aligned box of `size` (sx, sy, sz) standing on y = center_base.y,
    rotated about the vertical axis through its centre; outward winding."""
    sx, sy, sz = size
    x0, x1 = -sx / 2, sx / 2
    y0, y1 = 0.0, sy
    z0, z1 = -sz / 2, sz / 2
    c = [
        (x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0),
        (x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1),
    ]
    faces = [
        (0, 3, 2, 1),  # -z
        (4, 5, 6, 7),  # +z
        (0, 4, 7, 3),  # -x
        (1, 2, 6, 5),  # +x
        (0, 1, 5, 4),  # -y
        (3, 7, 6, 2),  # +y
    ]
    v = np.array(c, dtype=np.float64)
    a = math.radians(rot_y_deg)
    rot = np.array([[math.cos(a), 0, math.sin(a)], [0, 1, 0], [-math.sin(a), 0, math.cos(a)]])
    v = v @ rot.T + np.asarray(center_base, dtype=np.float64)
    tris = []
    for f in faces:
        tris.append([f[0], f[1], f[2]])
        tris.append([f[0], f[2], f[3]])
    return v, np.array(tris, dtype=np.uint32)


def centered_box(center, half_extent):
    """Closed axis-aligned box [center - h, center + h] with outward winding (12 triangles)."""
    h = np.broadcast_to(np.asarray(half_extent, dtype=np.float64), (3,))
    v, t = box_mesh(2 * h, (0.0, 0.0, 0.0), 0.0)
    v = v + np.asarray(center, dtype=np.float64) - np.array([0.0, h[1], 0.0])
    return v, t


def cornell_box(xres=256, yres=256, one_light_triangle=False) -> Scene:
    """Unit-cube Cornell box: 5 walls as 2-triangle quads (open towards the camera at
    z = 0), Lambert 0.75 white floor/ceiling/back wall, red left wall (0.75 in the bins
    centred at >= 605 nm, 0.05 elsewhere), green right wall (0.75 for 505-565 nm), a
    0.25 x 0.25 downward-facing area light just below the ceiling with flat emission 10,
    a 0.3^3 box at (0.65, 0, 0.35) rotated 17 degrees and a 0.3 x 0.6 x 0.3 box at
    (0.3, 0, 0.65) rotated -17 degrees.  Pinhole camera at (0.5, 0.5, -1.4) looking +z
    with a 40 degree field of view.  one_light_triangle keeps only the first triangle of
    the light quad: a scene with exactly one light, whose selection probability is 1."""
    s = Scene()
    s.name = "cornell_box"
    white = s.add_material(diffuse(0.75))
    red = s.add_material(diffuse(band_spectrum(0.75, 0.05, 23, 35)))
    green = s.add_material(diffuse(band_spectrum(0.75, 0.05, 13, 19)))
    light = s.add_material(area_light(10.0, reflectance=0.0))
    boxes = s.add_material(diffuse(0.75))
    # Walls with inward-facing winding normals.
    s.add_mesh(*quad((0, 0, 0), (0, 0, 1), (1, 0, 1), (1, 0, 0)), white)      # floor, +y
    s.add_mesh(*quad((0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1)), white)      # ceiling, -y
    s.add_mesh(*quad((0, 0, 1), (0, 1, 1), (1, 1, 1), (1, 0, 1)), white)      # back, -z
    s.add_mesh(*quad((0, 0, 0), (0, 1, 0), (0, 1, 1), (0, 0, 1)), red)        # left x=0, +x
    s.add_mesh(*quad((1, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0)), green)      # right x=1, -x
    q = 0.125
    yl = 1.0 - 1e-4
    lv, lt = quad((0.5 - q, yl, 0.5 - q), (0.5 + q, yl, 0.5 - q), (0.5 + q, yl, 0.5 + q), (0.5 - q, yl, 0.5 + q))
    s.add_mesh(lv, lt[:1] if one_light_triangle else lt, light)
    s.add_mesh(*box_mesh((0.3, 0.3, 0.3), (0.65, 0.0, 0.35), 17.0), boxes)
    s.add_mesh(*box_mesh((0.3, 0.6, 0.3), (0.3, 0.0, 0.65), -17.0), boxes)
    s.camera = CameraSpec(kind=abi.CAMERA_PINHOLE, pos=(0.5, 0.5, -1.4), dir=(0, 0, 1), up=(0, 1, 0),
                          fov_deg=40.0, xres=xres, yres=yres)
    return s


def cornell_box_materials(xres=64, yres=64) -> Scene:
    """The Cornell box with the tall box turned into glass and the small box into a
    rough Beckmann metal, a mirror back wall and a rough-glass sphere above the small box:
    exercises every shader; the floor is a dense dielectric (a smooth coating over a Lambert
    base)."""
    s = Scene()
    s.name = "cornell_box_materials"
    white = s.add_material(diffuse(0.75))
    red = s.add_material(diffuse(band_spectrum(0.75, 0.05, 23, 35)))
    green = s.add_material(diffuse(band_spectrum(0.75, 0.05, 13, 19)))
    light = s.add_material(area_light(10.0, reflectance=0.0))
    glass_m = s.add_material(glass(1.5))
    metal = s.add_material(microfacet(rgb_to_spectrum((0.9, 0.7, 0.4)), 0.2))
    mir = s.add_material(mirror(0.9))
    coated = s.add_material(dense_dielectric(0.1, 0.7))
    s.add_mesh(*quad((0, 0, 0), (0, 0, 1), (1, 0, 1), (1, 0, 0)), coated)
    s.add_mesh(*quad((0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1)), white)
    s.add_mesh(*quad((0, 0, 1), (0, 1, 1), (1, 1, 1), (1, 0, 1)), mir)
    s.add_mesh(*quad((0, 0, 0), (0, 1, 0), (0, 1, 1), (0, 0, 1)), red)
    s.add_mesh(*quad((1, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0)), green)
    q = 0.125
    yl = 1.0 - 1e-4
    s.add_mesh(*quad((0.5 - q, yl, 0.5 - q), (0.5 + q, yl, 0.5 - q), (0.5 + q, yl, 0.5 + q), (0.5 - q, yl, 0.5 + q)), light)
    s.add_mesh(*box_mesh((0.3, 0.3, 0.3), (0.65, 0.0, 0.35), 17.0), metal)
    s.add_mesh(*box_mesh((0.3, 0.6, 0.3), (0.3, 0.0, 0.65), -17.0), glass_m)
    s.add_sphere((0.65, 0.45, 0.35), 0.12, s.add_material(glossy_glass(1.5, 0.15)))
    s.camera = CameraSpec(kind=abi.CAMERA_PINHOLE, pos=(0.5, 0.5, -1.4), dir=(0, 0, 1), up=(0, 1, 0),
                          fov_deg=40.0, xres=xres, yres=yres)
    return s


def cornell_box_medium(xres=256, yres=256, one_light_triangle=False) -> Scene:
    """The Cornell box filled with a homogeneous chromatic medium: sigma_s rising linearly
    from 0.5 to 2.0 per unit across the 36 bins, sigma_a = 0.1, Henyey-Greenstein g = 0.7.
    The medium's boundary is a closed box 1e-3 outside the walls, so no wall coincides
    with it; rays leave the medium through the open side of the box."""
    s = cornell_box(xres, yres, one_light_triangle)
    s.name = "cornell_box_medium"
    sigma_s = 0.5 + 1.5 * np.arange(36) / 35.0
    med = s.add_medium(MediumSpec(sigma_s=sigma_s, sigma_a=np.full(36, 0.1), phase=abi.PHASE_HENYEY_GREENSTEIN,
                                  phase_g=0.7, priority=1))
    bnd = s.add_material(volume_boundary(med))
    e = 1e-3
    s.add_mesh(*centered_box((0.5, 0.5, 0.5), 0.5 + e), bnd)
    return s


def cornell_box_media_mix(xres=64, yres=64) -> Scene:
    """The Cornell box and its camera inside a thin fog (sigma_s 0.1, sigma_a 0.02,
    isotropic, priority 1, box from (-0.2, -0.2, -1.6) to (1.2, 1.2, 1.2)), with a glass
    sphere of radius 0.15 at (0.65, 0.5, 0.35) filled with a dense Rayleigh medium
    (sigma_s 3.0, sigma_a 0.5, priority 3: the glass surface itself changes the medium), and
    a purely absorbing chromatic box (sigma_a 4.0 in the long-wavelength half, 0.5 below,
    priority 2) of half size 0.1 at (0.5, 0.75, 0.6)."""
    s = cornell_box(xres, yres)
    s.name = "cornell_box_media_mix"
    fog = s.add_medium(MediumSpec(sigma_s=np.full(36, 0.1), sigma_a=np.full(36, 0.02), priority=1))
    dense = s.add_medium(MediumSpec(sigma_s=np.full(36, 3.0), sigma_a=np.full(36, 0.5),
                                    phase=abi.PHASE_RAYLEIGH, priority=3))
    absorb = s.add_medium(MediumSpec(sigma_s=np.zeros(36), sigma_a=band_spectrum(4.0, 0.5, 18, 35), priority=2))
    lo, hi = np.array([-0.2, -0.2, -1.6]), np.array([1.2, 1.2, 1.2])
    s.add_mesh(*centered_box((lo + hi) / 2, (hi - lo) / 2), s.add_material(volume_boundary(fog)))
    g = glass(1.5)
    g.medium_inside = dense
    v, t = icosphere(3)
    s.add_mesh(v * 0.15 + np.array([0.65, 0.5, 0.35]), t, s.add_material(g))
    s.add_mesh(*centered_box((0.5, 0.75, 0.6), 0.1), s.add_material(volume_boundary(absorb)))
    return s


# --------------------------------------------------------------------------------------
def icosphere(level: int):
    """Unit icosphere: 20 * 4**level triangles, outward winding, shared vertices."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = np.array(v, dtype=np.float64)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    faces = np.array(f, dtype=np.int64)
    for _ in range(level):
        nv = len(verts)
        e = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
        e.sort(axis=1)
        keys = e[:, 0] * (nv + 1) + e[:, 1]
        uniq, inv = np.unique(keys, return_inverse=True)
        a = uniq // (nv + 1)
        b = uniq % (nv + 1)
        mid = verts[a] + verts[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        verts = np.concatenate([verts, mid])
        nf = len(faces)
        m01 = nv + inv[:nf]
        m12 = nv + inv[nf:2 * nf]
        m20 = nv + inv[2 * nf:]
        v0, v1, v2 = faces[:, 0], faces[:, 1], faces[:, 2]
        faces = np.concatenate([
            np.stack([v0, m01, m20], 1), np.stack([v1, m12, m01], 1),
            np.stack([v2, m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return verts, faces.astype(np.uint32)


def fbm_heightfield(n: int, octaves: int, rng: np.random.Generator) -> np.ndarray:
    """n x n fractional Brownian motion from value noise: octave k has a (2^(k+2)+1)^2
    random lattice interpolated bilinearly, amplitude 0.5^k; normalised to [-1, 1]."""
    h = np.zeros((n, n))
    xs = np.linspace(0.0, 1.0, n)
    amp = 1.0
    for k in range(octaves):
        cells = 2 ** (k + 2)
        lat = rng.uniform(-1.0, 1.0, size=(cells + 1, cells + 1))
        g = xs * cells
        i = np.minimum(g.astype(np.int64), cells - 1)
        f = g - i
        f = f * f * (3 - 2 * f)
        a = lat[np.ix_(i, i)]
        b = lat[np.ix_(i + 1, i)]
        c = lat[np.ix_(i, i + 1)]
        d = lat[np.ix_(i + 1, i + 1)]
        fx = f[:, None]
        fz = f[None, :]
        h += amp * ((a * (1 - fx) + b * fx) * (1 - fz) + (c * (1 - fx) + d * fx) * fz)
        amp *= 0.5
    h -= h.min()
    h /= max(h.max(), 1e-12)
    return 2.0 * h - 1.0


def sky_texture(width: int, height: int) -> np.ndarray:
    """Equirect float32 RGB sky: deep blue at the zenith fading to a pale horizon, and a
    dim ground below the horizon.  Row 0 is the zenith (EnvMapLight convention)."""
    theta = (np.arange(height) + 0.5) / height * np.pi  # 0 = zenith
    elev = np.pi / 2 - theta
    tex = np.zeros((height, width, 3), dtype=np.float32)
    zen = np.array([0.10, 0.25, 0.80])
    hor = np.array([0.70, 0.80, 0.95])
    gnd = np.array([0.25, 0.22, 0.20])
    up = np.clip(elev / (np.pi / 2), 0, 1)[:, None]
    col = np.where(elev[:, None] >= 0, hor * (1 - up) + zen * up, gnd * np.ones_like(up))
    tex[:] = col[:, None, :].astype(np.float32)
    return tex


def terrain_spheres(xres=1920, yres=1080, terrain_n=1024, sphere_level=5, num_spheres=32,
                    env_w=2048, env_h=1024, seed=1) -> Scene:
    rng = np.random.default_rng(seed)
    s = Scene()
    s.name = "terrain_spheres"
    extent = 10.0
    amp = 0.2
    hf = amp * fbm_heightfield(terrain_n, 6, rng)
    xs = np.linspace(-extent / 2, extent / 2, terrain_n)
    X, Z = np.meshgrid(xs, xs, indexing="ij")
    verts = np.stack([X, hf, Z], axis=-1).reshape(-1, 3)
    # Smooth normals from central differences.
    dx = extent / (terrain_n - 1)
    gx = np.gradient(hf, dx, axis=0)
    gz = np.gradient(hf, dx, axis=1)
    nrm = np.stack([-gx, np.ones_like(hf), -gz], axis=-1)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    idx = np.arange(terrain_n * terrain_n, dtype=np.int64).reshape(terrain_n, terrain_n)
    a = idx[:-1, :-1].ravel()
    b = idx[1:, :-1].ravel()
    c = idx[1:, 1:].ravel()
    d = idx[:-1, 1:].ravel()
    # Upward winding: (b - a) x (c - a) has +y for x increasing along i, z along j.
    tris = np.concatenate([np.stack([a, d, c], 1), np.stack([a, c, b], 1)]).astype(np.uint32)
    ground = s.add_material(diffuse(rgb_to_spectrum((0.35, 0.30, 0.22))))
    s.add_mesh(verts, tris, ground, normals=nrm.reshape(-1, 3))
    sv, sf = icosphere(sphere_level)
    kinds = np.array([0] * 13 + [1] * 10 + [2] * 9)[:num_spheres]
    rng.shuffle(kinds)
    for k in range(num_spheres):
        r = rng.uniform(0.1, 0.4)
        px, pz = rng.uniform(-4.0, 4.0, size=2)
        i = int(round((px + extent / 2) / dx))
        j = int(round((pz + extent / 2) / dx))
        py = hf[min(max(i, 0), terrain_n - 1), min(max(j, 0), terrain_n - 1)] + r
        if kinds[k] == 0:
            alb = rng.uniform(0.2, 0.8, size=3)
            m = s.add_material(diffuse(rgb_to_spectrum(alb)))
        elif kinds[k] == 1:
            rough = rng.uniform(0.05, 0.5)
            tint = rng.uniform(0.5, 0.95, size=3)
            m = s.add_material(microfacet(rgb_to_spectrum(tint), rough))
        else:
            m = s.add_material(glass(1.5))
        s.add_mesh(sv * r + np.array([px, py, pz]), sf, m, normals=sv)
    s.env_lights.append(env_map(sky_texture(env_w, env_h), up=(0.0, 1.0, 0.0)))
    elev = math.radians(35.0)
    az = math.radians(30.0)
    dir_out = (-math.cos(elev) * math.cos(az), -math.sin(elev), -math.cos(elev) * math.sin(az))
    s.env_lights.append(sun_light(100.0, dir_out, 0.265))
    s.camera = CameraSpec(kind=abi.CAMERA_PINHOLE, pos=(0.0, 2.2, -6.5), dir=(0.0, -0.3, 1.0), up=(0, 1, 0),
                          fov_deg=60.0, xres=xres, yres=yres)
    return s


def terrain_spheres_small(xres=96, yres=54) -> Scene:
    """Scaled-down terrain scene (same generator) for parity tests."""
    return terrain_spheres(xres=xres, yres=yres, terrain_n=64, sphere_level=2, num_spheres=8, env_w=128, env_h=64)


# --------------------------------------------------------------------------------------
# Spheres and planetary atmospheres.
WAVELENGTHS_NM = 375.0 + 10.0 * np.arange(36)


def earth_atmosphere_table(h0=-1.0, dh=0.5, rows=403, rayleigh_680=5.8e-3, rayleigh_height=8.0, mie=2.0e-2,
                           mie_height=1.2, ozone_peak=2.5e-3, ozone_altitude=25.0, ozone_width=8.0):
    """Collision coefficients per km at altitudes h0 + i * dh (the row layout of the
    reference's earth_atmosphere_collision_coefficients.json): Rayleigh scattering
    5.8e-6 /m at 680 nm scaled as lambda^-4 with an 8 km scale height; Mie scattering
    2e-5 /m with a 1.2 km scale height; ozone absorption with a Gaussian altitude profile
    peaking at 25 km and a Gaussian Chappuis band centred at 600 nm.  Returns
    (sigma_t, sigma_s_molecules, sigma_s_aerosols), each (rows, 36)."""
    h = h0 + dh * np.arange(rows)
    lam = WAVELENGTHS_NM
    mol = rayleigh_680 * (680.0 / lam)[None, :] ** 4 * np.exp(-h / rayleigh_height)[:, None]
    aer = mie * np.exp(-h / mie_height)[:, None] * np.ones((1, 36))
    ozone = ozone_peak * np.exp(-(((h - ozone_altitude) / ozone_width) ** 2))[:, None] * \
        np.exp(-(((lam - 600.0) / 60.0) ** 2))[None, :]
    return mol + aer + ozone, mol, aer


def simple_atmosphere_table(h0=-1.0, dh=0.05, rows=4021):
    """The reference's ExponentialConstituentDistribution (atmosphere.cxx:127-188)
    tabulated: molecular Rayleigh scattering from the refractive index of air
    (n = 1.00028, 1.225 kg/m^3 of 29 g/mol) with an 8 km scale height; aerosols with
    sigma_s 20e-3 /km and sigma_a 2.22e-3 /km at sea level and a 1.2 km scale height."""
    h = h0 + dh * np.arange(rows)
    n_air = 1.225 * 6.022e23 / 29e-3
    prefactor = 8.0 * math.pi ** 3 / 3.0 * (1.00028 ** 2 - 1.0) ** 2 / n_air * 1e27 * 1e12
    mol = (prefactor / WAVELENGTHS_NM ** 4)[None, :] * np.exp(-h / 8.0)[:, None]
    aer_s = 20e-3 * np.exp(-h / 1.2)[:, None] * np.ones((1, 36))
    aer_a = 2.22e-3 * np.exp(-h / 1.2)[:, None] * np.ones((1, 36))
    return mol + aer_s + aer_a, mol, aer_s


def planet_atmosphere(xres=64, yres=64, radius=6371.0, camera_height=0.002, sun_elevation_deg=10.0, g=0.76,
                      table=None, h0=-1.0, dh=0.5, camera_kind=abi.CAMERA_FISHEYE, ground_albedo=0.3,
                      sun_power=20.0) -> Scene:
    """A spherical planet (radius in km) under a tabulated atmosphere, lit by the sun at
    `sun_elevation_deg` above the horizon of the camera, which stands `camera_height` km
    above the ground looking up (fisheye by default).  The ground is an analytic sphere
    with a Lambert albedo; the atmosphere's boundary is a concentric sphere at the top of
    the table."""
    s = Scene()
    s.name = "planet_atmosphere"
    tab = earth_atmosphere_table(h0=h0, dh=dh) if table is None else table
    atm = AtmosphereSpec(planet_center=(0.0, 0.0, 0.0), planet_radius=radius, h0=h0, dh=dh, sigma_t=tab[0],
                         sigma_s_molecules=tab[1], sigma_s_aerosols=tab[2], g=g, priority=1)
    mid = s.add_medium(atm)
    s.add_sphere((0.0, 0.0, 0.0), radius, s.add_material(diffuse(ground_albedo)))
    s.add_sphere((0.0, 0.0, 0.0), radius + atm.top_altitude, s.add_material(volume_boundary(mid)))
    e = math.radians(sun_elevation_deg)
    s.env_lights.append(sun_light(sun_power, (-math.cos(e), -math.sin(e), 0.0), 0.265))
    s.camera = CameraSpec(kind=camera_kind, pos=(0.0, radius + camera_height, 0.0), dir=(0.0, 1.0, 0.0),
                          up=(0.0, 0.0, 1.0), fov_deg=90.0, xres=xres, yres=yres)
    return s


def planet_from_space(xres=64, yres=64, distance=5.0) -> Scene:
    """The planet of planet_atmosphere seen from `distance` planet radii away with a 30
    degree pinhole camera: rays enter the atmosphere from empty space."""
    s = planet_atmosphere(xres, yres, camera_kind=abi.CAMERA_PINHOLE)
    s.name = "planet_from_space"
    R = 6371.0
    s.camera = CameraSpec(kind=abi.CAMERA_PINHOLE, pos=(-distance * R * 0.8, distance * R * 0.6, 0.0),
                          dir=(0.8, -0.6, 0.0), up=(0.0, 0.0, 1.0), fov_deg=30.0, xres=xres, yres=yres)
    return s


def spheres_box(xres=64, yres=64) -> Scene:
    """The Cornell box with analytic spheres: a mirror sphere, a glass sphere filled with
    a homogeneous medium, a diffuse sphere, and a small emissive sphere as a second light."""
    s = cornell_box(xres, yres)
    s.name = "spheres_box"
    s.add_sphere((0.25, 0.15, 0.3), 0.15, s.add_material(mirror(0.9)))
    g = glass(1.5)
    g.medium_inside = s.add_medium(MediumSpec(sigma_s=np.full(36, 2.0), sigma_a=band_spectrum(1.5, 0.2, 0, 17),
                                              phase=abi.PHASE_HENYEY_GREENSTEIN, phase_g=0.5, priority=1))
    s.add_sphere((0.72, 0.45, 0.35), 0.12, s.add_material(g))
    s.add_sphere((0.55, 0.1, 0.75), 0.1, s.add_material(diffuse(rgb_to_spectrum((0.2, 0.4, 0.8)))))
    s.add_sphere((0.2, 0.8, 0.5), 0.04, s.add_material(area_light(30.0)))
    return s


def guiding_room(xres=1280, yres=720, emission=60.0) -> Scene:
    """The guiding workload: a 4 x 3 x 4 room (x, y up, z) with Lambert 0.6 walls and ceiling
    and a glossy Beckmann floor (reflectance 0.5, alpha 0.1), lit only by an area light
    outside: a 1 x 1 quad (flat emission `emission`) 0.6 behind a 0.3 x 0.3 gap in the wall at
    x = 4, facing it.  The light enters as one beam through the gap, so almost every point of
    the room is lit indirectly from the beam's patch, which BSDF sampling finds rarely and a
    learned guide can point at.  Pinhole camera at (3.7, 1.6, 0.4) looking at (0, 0.8, 3) with
    a 75 degree field of view (the gap is behind it)."""
    s = Scene()
    s.name = "guiding_room"
    wall = s.add_material(diffuse(0.6))
    floor = s.add_material(microfacet(0.5, 0.1))
    light = s.add_material(area_light(emission, reflectance=0.0))
    X, Y, Z = 4.0, 3.0, 4.0
    s.add_mesh(*quad((0, 0, 0), (0, 0, Z), (X, 0, Z), (X, 0, 0)), floor)
    s.add_mesh(*quad((0, Y, 0), (X, Y, 0), (X, Y, Z), (0, Y, Z)), wall)
    s.add_mesh(*quad((0, 0, 0), (0, Y, 0), (0, Y, Z), (0, 0, Z)), wall)          # x = 0
    s.add_mesh(*quad((0, 0, 0), (X, 0, 0), (X, Y, 0), (0, Y, 0)), wall)          # z = 0
    s.add_mesh(*quad((0, 0, Z), (0, Y, Z), (X, Y, Z), (X, 0, Z)), wall)          # z = 4
    # Wall x = X around the gap y in [1.35, 1.65], z in [1.85, 2.15].
    y0, y1, z0, z1 = 1.35, 1.65, 1.85, 2.15
    s.add_mesh(*quad((X, 0, 0), (X, y0, 0), (X, y0, Z), (X, 0, Z)), wall)
    s.add_mesh(*quad((X, y1, 0), (X, Y, 0), (X, Y, Z), (X, y1, Z)), wall)
    s.add_mesh(*quad((X, y0, 0), (X, y1, 0), (X, y1, z0), (X, y0, z0)), wall)
    s.add_mesh(*quad((X, y0, z1), (X, y1, z1), (X, y1, Z), (X, y0, Z)), wall)
    # Light outside at x = X + 0.6 facing -x (winding normal (p1 - p0) x (p2 - p0) = -x).
    xl = X + 0.6
    s.add_mesh(*quad((xl, 1.0, 1.5), (xl, 1.0, 2.5), (xl, 2.0, 2.5), (xl, 2.0, 1.5)), light)
    s.camera = CameraSpec(kind=abi.CAMERA_PINHOLE, pos=(3.7, 1.6, 0.4), dir=(-3.7, -0.8, 2.6), up=(0, 1, 0),
                          fov_deg=75.0, xres=xres, yres=yres)
    return s


VIEW_RESOLUTIONS = (128, 256, 512, 768, 1024)


def terrain_views(n=96, seed=4, spp_range=(4, 64), resolutions=VIEW_RESOLUTIONS):
    """The multi-view workload: n seeded camera poses over the terrain_spheres scene, each
    a square view with its side drawn uniformly from `resolutions` and its samples per pixel
    uniformly from spp_range (inclusive).  Cameras sit 0.8-3.0 above the terrain within the
    central 8 x 8 and look at a point near the centre.  Returns [(CameraSpec, spp)]."""
    rng = np.random.default_rng(seed)
    views = []
    for _ in range(n):
        side = int(rng.choice(resolutions))
        spp = int(rng.integers(spp_range[0], spp_range[1] + 1))
        pos = np.array([rng.uniform(-4, 4), rng.uniform(0.8, 3.0), rng.uniform(-4, 4)])
        target = np.array([rng.uniform(-2, 2), 0.0, rng.uniform(-2, 2)])
        d = target - pos
        if np.linalg.norm(d[[0, 2]]) < 0.5:
            d[0] += 1.0
        views.append((CameraSpec(kind=abi.CAMERA_PINHOLE, pos=tuple(pos), dir=tuple(d / np.linalg.norm(d)),
                                 up=(0.0, 1.0, 0.0), fov_deg=float(rng.uniform(40, 75)), xres=side, yres=side), spp))
    return views
