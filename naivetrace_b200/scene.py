"""Host-side scene model: the Scene / Material / light / camera objects of the reference
(src/scene.hxx:134-315, src/light.hxx, src/camera.hxx) reduced to what the forward path
tracer consumes, and their flattening into the C-ABI's tt_scene_desc.

Geometry is stored the way the reference's Mesh stores it (float32 vertices, uint32 index
triples, optional per-vertex normals, primitive.hxx:59-88).  Triangles keep the order in
which they were added; that order defines the global primitive ids reported by the
intersection entry points.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import abi
from .spectral import as_spectrum

NBINS = abi.NBINS


@dataclass
class MaterialSpec:
    """Shader + optional UniformAreaLight (struct Material, scene.hxx:45-54)."""

    shader: int = abi.SHADER_DIFFUSE
    reflectance: np.ndarray = field(default_factory=lambda: np.full(NBINS, 0.8))
    alpha: float = 0.0
    ior_ratio: float = 1.5
    emission: Optional[np.ndarray] = None
    medium_inside: int = -1
    medium_outside: int = -1
    volume_boundary: bool = False
    diffuse_texture: int = -1  # index of the scene texture multiplying the diffuse reflectance
    specular_reflectivity: float = 0.0  # dense dielectric coating at normal incidence

    def to_c(self) -> abi.Material:
        m = abi.Material()
        m.shader = int(self.shader)
        m.reflectance[:] = [float(x) for x in as_spectrum(self.reflectance)]
        m.alpha = float(self.alpha)
        m.ior_ratio = float(self.ior_ratio)
        if self.emission is not None:
            m.emissive = 1
            m.emission[:] = [float(x) for x in as_spectrum(self.emission)]
        m.medium_inside = int(self.medium_inside) + 1  # C ABI: 0 = none, k = medium k-1
        m.medium_outside = int(self.medium_outside) + 1
        m.volume_boundary = int(bool(self.volume_boundary))
        m.diffuse_texture = int(self.diffuse_texture) + 1  # C ABI: 0 = none, k = texture k-1
        m.specular_reflectivity = float(self.specular_reflectivity)
        return m


@dataclass
class MediumSpec:
    """HomogeneousMedium (shader.cxx:1234-1316) with its phase function."""

    sigma_s: np.ndarray
    sigma_a: np.ndarray
    phase: int = abi.PHASE_UNIFORM
    phase_g: float = 0.0
    priority: int = 1

    def to_c(self, keep: list) -> abi.Medium:
        m = abi.Medium()
        m.kind = abi.MEDIUM_HOMOGENEOUS
        m.priority = int(self.priority)
        m.sigma_s[:] = [float(x) for x in as_spectrum(self.sigma_s)]
        m.sigma_a[:] = [float(x) for x in as_spectrum(self.sigma_a)]
        m.phase = int(self.phase)
        m.phase_g = float(self.phase_g)
        return m


@dataclass
class AtmosphereSpec:
    """Atmosphere::Tabulated (atmosphere.cxx:234-348 with SphereGeometry,
    atmosphere.hxx:95-123), lengths in km: rows of sigma_t, sigma_s of molecules (Rayleigh
    phase) and of aerosols (Henyey-Greenstein g) per km at altitudes h0 + i * dh."""

    planet_center: tuple
    planet_radius: float
    h0: float
    dh: float
    sigma_t: np.ndarray            # (n, 36)
    sigma_s_molecules: np.ndarray  # (n, 36)
    sigma_s_aerosols: np.ndarray   # (n, 36)
    g: float = 0.7
    priority: int = 1

    @property
    def top_altitude(self) -> float:
        return self.h0 + self.dh * (len(self.sigma_t) - 1)

    def to_c(self, keep: list) -> abi.Medium:
        m = abi.Medium()
        m.kind = abi.MEDIUM_ATMOSPHERE
        m.priority = int(self.priority)
        m.phase = abi.PHASE_HENYEY_GREENSTEIN
        m.phase_g = float(self.g)
        m.planet_center[:] = [float(x) for x in self.planet_center]
        m.planet_radius = float(self.planet_radius)
        tabs = [np.ascontiguousarray(a, dtype=np.float32).reshape(-1, NBINS)
                for a in (self.sigma_t, self.sigma_s_molecules, self.sigma_s_aerosols)]
        if not (len(tabs[0]) == len(tabs[1]) == len(tabs[2]) >= 2):
            raise ValueError("atmosphere tables need the same number (>= 2) of altitude rows")
        keep.extend(tabs)
        m.table_size = len(tabs[0])
        m.table_h0 = float(self.h0)
        m.table_dh = float(self.dh)
        m.sigma_t, m.sigma_s_molecules, m.sigma_s_aerosols = [t.ctypes.data_as(C.POINTER(C.c_float)) for t in tabs]
        return m


def volume_boundary(medium_inside: int, medium_outside: int = -1) -> MaterialSpec:
    """Invisible triangles that only delimit media (a material without shader)."""
    return MaterialSpec(shader=abi.SHADER_DIFFUSE, reflectance=np.zeros(NBINS), medium_inside=medium_inside,
                        medium_outside=medium_outside, volume_boundary=True)


def diffuse(reflectance) -> MaterialSpec:
    return MaterialSpec(shader=abi.SHADER_DIFFUSE, reflectance=as_spectrum(reflectance))


def mirror(reflectance) -> MaterialSpec:
    return MaterialSpec(shader=abi.SHADER_SPECULAR_REFLECTIVE, reflectance=as_spectrum(reflectance))


def glass(ior_ratio: float) -> MaterialSpec:
    return MaterialSpec(shader=abi.SHADER_SPECULAR_DIELECTRIC, reflectance=np.zeros(NBINS), ior_ratio=ior_ratio)


def microfacet(reflectance, alpha: float) -> MaterialSpec:
    return MaterialSpec(shader=abi.SHADER_MICROFACET, reflectance=as_spectrum(reflectance), alpha=alpha)


def glossy_glass(ior_ratio: float, alpha: float) -> MaterialSpec:
    """GlossyTransmissiveDielectricShader (shader.cxx:710-787): a rough dielectric interface."""
    return MaterialSpec(shader=abi.SHADER_GLOSSY_DIELECTRIC, reflectance=np.zeros(NBINS), ior_ratio=ior_ratio,
                        alpha=alpha)


def dense_dielectric(specular_reflectivity: float, diffuse_reflectance) -> MaterialSpec:
    """SpecularDenseDielectricShader (shader.cxx:977-1081): a smooth coating over a Lambert base."""
    return MaterialSpec(shader=abi.SHADER_SPECULAR_DENSE_DIELECTRIC, reflectance=as_spectrum(diffuse_reflectance),
                        specular_reflectivity=specular_reflectivity)


def area_light(emission, reflectance=0.0) -> MaterialSpec:
    return MaterialSpec(shader=abi.SHADER_DIFFUSE, reflectance=as_spectrum(reflectance), emission=as_spectrum(emission))


@dataclass
class EnvLightSpec:
    kind: int
    spectrum: np.ndarray = field(default_factory=lambda: np.zeros(NBINS))
    dir: tuple = (0.0, 1.0, 0.0)
    scalar: float = 0.0
    scalar2: float = 0.0
    texture: Optional[np.ndarray] = None  # (h, w, 3) float32, row 0 = top


def dome_light(spectrum, up=(0.0, 1.0, 0.0)) -> EnvLightSpec:
    return EnvLightSpec(kind=abi.ENV_DOME, spectrum=as_spectrum(spectrum), dir=tuple(up))


def sun_light(total_power: float, dir_out, opening_angle_deg: float) -> EnvLightSpec:
    """Sun (light.hxx:238-288).  dir_out: direction the light travels.  The opening angle
    is the half angle of the cone of directions that receive light."""
    return EnvLightSpec(kind=abi.ENV_SUN, dir=tuple(dir_out), scalar=total_power, scalar2=opening_angle_deg)


def env_map(texture: np.ndarray, up=(0.0, 1.0, 0.0)) -> EnvLightSpec:
    tex = np.ascontiguousarray(texture, dtype=np.float32)
    assert tex.ndim == 3 and tex.shape[2] == 3
    return EnvLightSpec(kind=abi.ENV_MAP, dir=tuple(up), texture=tex)


def directional_light(spectrum, dir_out) -> EnvLightSpec:
    return EnvLightSpec(kind=abi.ENV_DIRECTIONAL, spectrum=as_spectrum(spectrum), dir=tuple(dir_out))


@dataclass
class CameraSpec:
    kind: int = abi.CAMERA_PINHOLE
    pos: tuple = (0.0, 0.0, 0.0)
    dir: tuple = (0.0, 0.0, 1.0)
    up: tuple = (0.0, 1.0, 0.0)
    fov_deg: float = 40.0
    xres: int = 64
    yres: int = 64

    @property
    def num_pixels(self) -> int:
        return self.xres * self.yres

    def to_c(self) -> abi.Camera:
        c = abi.Camera()
        c.kind = self.kind
        c.pos[:] = [float(x) for x in self.pos]
        c.dir[:] = [float(x) for x in self.dir]
        c.up[:] = [float(x) for x in self.up]
        c.fov_deg = float(self.fov_deg)
        c.xres = int(self.xres)
        c.yres = int(self.yres)
        return c


class Scene:
    """Triangle soup with per-triangle material, lights and one camera."""

    def __init__(self):
        self._verts: List[np.ndarray] = []
        self._norms: List[Optional[np.ndarray]] = []
        self._tris: List[np.ndarray] = []
        self._mats_of_tris: List[np.ndarray] = []
        self._uvs: List[Optional[np.ndarray]] = []
        self.textures: List[np.ndarray] = []  # linear RGB float32, (height, width, 3), row 0 at the top
        self._nverts = 0
        self.materials: List[MaterialSpec] = []
        self.env_lights: List[EnvLightSpec] = []
        self.point_lights: List[tuple] = []
        self.media: list = []  # MediumSpec or AtmosphereSpec
        self._spheres: List[tuple] = []  # (cx, cy, cz, r, material)
        self.camera = CameraSpec()
        self.name = "scene"
        self._flat = None

    # -- building -----------------------------------------------------------------
    def add_material(self, m: MaterialSpec) -> int:
        self.materials.append(m)
        self._flat = None
        return len(self.materials) - 1

    def add_medium(self, m) -> int:
        self.media.append(m)
        return len(self.media) - 1

    def add_sphere(self, center, radius: float, material: int) -> int:
        """Analytic sphere (Spheres, primitive.hxx:94-136); returns its global primitive id
        (spheres are numbered after all triangles)."""
        self._spheres.append((float(center[0]), float(center[1]), float(center[2]), float(radius), int(material)))
        return len(self._spheres) - 1

    @property
    def num_spheres(self) -> int:
        return len(self._spheres)

    def sphere_arrays(self):
        if not self._spheres:
            return np.zeros((0, 4), np.float32), np.zeros(0, np.uint32)
        a = np.array(self._spheres, dtype=np.float64)
        return np.ascontiguousarray(a[:, :4], dtype=np.float32), np.ascontiguousarray(a[:, 4], dtype=np.uint32)

    def add_texture(self, rgb) -> int:
        """A diffuse texture (linear RGB, (height, width, 3), row 0 at the top); returns its index."""
        t = np.ascontiguousarray(rgb, dtype=np.float32)
        if t.ndim != 3 or t.shape[2] != 3 or t.shape[0] < 1 or t.shape[1] < 1:
            raise ValueError("a texture is a (height, width, 3) array")
        self.textures.append(t)
        return len(self.textures) - 1

    def add_mesh(self, vertices, triangles, material: int, normals=None, uvs=None) -> None:
        v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
        if t.size and int(t.max()) >= len(v):
            raise ValueError("triangle index out of range")
        self._uvs.append(None if uvs is None else np.ascontiguousarray(uvs, dtype=np.float32).reshape(-1, 2))
        if self._uvs[-1] is not None and len(self._uvs[-1]) != len(v):
            raise ValueError("one texture coordinate pair per vertex")
        self._verts.append(v)
        self._norms.append(None if normals is None else np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 3))
        self._tris.append(t + np.uint32(self._nverts))
        self._mats_of_tris.append(np.full(len(t), material, dtype=np.uint32))
        self._nverts += len(v)
        self._flat = None

    def add_point_light(self, spectrum, pos) -> None:
        self.point_lights.append((as_spectrum(spectrum), tuple(pos)))
        self._flat = None

    # -- flattening -----------------------------------------------------------------
    def arrays(self):
        if self._flat is None:
            verts = np.concatenate(self._verts) if self._verts else np.zeros((0, 3), np.float32)
            tris = np.concatenate(self._tris) if self._tris else np.zeros((0, 3), np.uint32)
            mats = np.concatenate(self._mats_of_tris) if self._mats_of_tris else np.zeros(0, np.uint32)
            if any(n is not None for n in self._norms):
                norms = []
                for v, n, t in zip(self._verts, self._norms, self._tris):
                    if n is None:
                        raise ValueError("either all meshes or none must carry normals")
                    norms.append(n)
                norms = np.ascontiguousarray(np.concatenate(norms))
            else:
                norms = None
            self._flat = (np.ascontiguousarray(verts), norms, np.ascontiguousarray(tris), np.ascontiguousarray(mats))
        return self._flat

    def uv_array(self):
        """Texture coordinates of all vertices (num_vertices, 2), zeros for meshes without;
        None when no mesh has any."""
        if all(u is None for u in self._uvs):
            return None
        return np.ascontiguousarray(np.concatenate(
            [u if u is not None else np.zeros((len(v), 2), np.float32) for v, u in zip(self._verts, self._uvs)]))

    @property
    def num_triangles(self) -> int:
        return int(sum(len(t) for t in self._tris))

    def bounding_box(self):
        v = self.arrays()[0].astype(np.float64)
        sph, _ = self.sphere_arrays()
        pts = [v]
        if len(sph):
            c, r = sph[:, :3].astype(np.float64), sph[:, 3:4].astype(np.float64)
            pts += [c - r, c + r]
        p = np.concatenate(pts)
        return p.min(axis=0), p.max(axis=0)

    def to_desc(self):
        """Returns (tt_scene_desc, keepalive).  keepalive owns every array the descriptor
        points to and must outlive its use."""
        verts, norms, tris, mats = self.arrays()
        keep = [verts, norms, tris, mats]
        d = abi.SceneDesc()
        d.num_vertices = len(verts)
        d.vertices = verts.ctypes.data_as(C.POINTER(C.c_float))
        d.normals = norms.ctypes.data_as(C.POINTER(C.c_float)) if norms is not None else None
        d.num_triangles = len(tris)
        d.indices = tris.ctypes.data_as(C.POINTER(C.c_uint32))
        d.material_ids = mats.ctypes.data_as(C.POINTER(C.c_uint32))
        mat_arr = (abi.Material * max(1, len(self.materials)))(*[m.to_c() for m in self.materials])
        keep.append(mat_arr)
        d.num_materials = len(self.materials)
        d.materials = C.cast(mat_arr, C.POINTER(abi.Material))
        envs = []
        for e in self.env_lights:
            c = abi.EnvLight()
            c.kind = e.kind
            c.spectrum[:] = [float(x) for x in as_spectrum(e.spectrum)]
            c.dir[:] = [float(x) for x in e.dir]
            c.scalar = float(e.scalar)
            c.scalar2 = float(e.scalar2)
            if e.texture is not None:
                tex = np.ascontiguousarray(e.texture, dtype=np.float32)
                keep.append(tex)
                c.tex_height, c.tex_width = int(tex.shape[0]), int(tex.shape[1])
                c.tex_rgb = tex.ctypes.data_as(C.POINTER(C.c_float))
            envs.append(c)
        env_arr = (abi.EnvLight * max(1, len(envs)))(*envs)
        keep.append(env_arr)
        d.num_env_lights = len(envs)
        d.env_lights = C.cast(env_arr, C.POINTER(abi.EnvLight))
        pts = []
        for spec, pos in self.point_lights:
            p = abi.PointLight()
            p.spectrum[:] = [float(x) for x in spec]
            p.pos[:] = [float(x) for x in pos]
            pts.append(p)
        pt_arr = (abi.PointLight * max(1, len(pts)))(*pts)
        keep.append(pt_arr)
        d.num_point_lights = len(pts)
        d.point_lights = C.cast(pt_arr, C.POINTER(abi.PointLight))
        med_arr = (abi.Medium * max(1, len(self.media)))(*[m.to_c(keep) for m in self.media])
        keep.append(med_arr)
        d.num_media = len(self.media)
        d.media = C.cast(med_arr, C.POINTER(abi.Medium))
        sph, smat = self.sphere_arrays()
        keep += [sph, smat]
        d.num_spheres = len(sph)
        d.spheres = sph.ctypes.data_as(C.POINTER(C.c_float)) if len(sph) else None
        d.sphere_material_ids = smat.ctypes.data_as(C.POINTER(C.c_uint32)) if len(sph) else None
        cam = self.camera
        d.camera.kind = cam.kind
        d.camera.pos[:] = [float(x) for x in cam.pos]
        d.camera.dir[:] = [float(x) for x in cam.dir]
        d.camera.up[:] = [float(x) for x in cam.up]
        d.camera.fov_deg = float(cam.fov_deg)
        d.camera.xres = int(cam.xres)
        d.camera.yres = int(cam.yres)
        uv = self.uv_array()
        keep.append(uv)
        d.uvs = uv.ctypes.data_as(C.POINTER(C.c_float)) if uv is not None else None
        texs = []
        for t in self.textures:
            tx = abi.Texture()
            tx.height, tx.width = int(t.shape[0]), int(t.shape[1])
            tx.rgb = t.ctypes.data_as(C.POINTER(C.c_float))
            texs.append(tx)
        tex_arr = (abi.Texture * max(1, len(texs)))(*texs)
        keep.append(tex_arr)
        d.num_textures = len(texs)
        d.textures = C.cast(tex_arr, C.POINTER(abi.Texture))
        return d, keep


def make_params(max_ray_depth: int = 25, pt_sample_mode: int = abi.SAMPLE_BOTH, max_spp: int = -1,
                wave_paths: int = 0, device: int = 0, algo: int = abi.ALGO_PT, qmc: bool = False,
                sort_shading: bool | None = None) -> abi.Params:
    """sort_shading: None = the library default (material-sorted shading from the second
    bounce on in scenes without media whose surfaces use three or more shader kinds),
    True = always sorted, False = traversal order."""
    p = abi.Params()
    p.sort_shading = 0 if sort_shading is None else (1 if sort_shading else -1)
    p.algo = algo
    p.qmc = int(bool(qmc))
    p.max_ray_depth = max_ray_depth
    p.pt_sample_mode = pt_sample_mode
    p.max_samples_per_pixel = max_spp
    p.wave_paths = wave_paths
    p.device = device
    return p
