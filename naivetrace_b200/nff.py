"""Reader for the reference's NFF scene files (the extended Neutral File Format of
src/parsenff.cxx:113-831) into a `Scene` for the CUDA tracer.

Directives (one per line, `#` comments; `{ ... }` opens a child scope that inherits and then
forgets the parent's transform, active shader / medium / area emitter and named
definitions):
  v | vfisheye + from/at/up/resolution[/angle]   pinhole (horizontal angle in degrees) or
                                                  fisheye camera
  transform [tx ty tz [h p b [sx sy sz]]]         translation, heading/pitch/bank (radians,
                                                  about y, x, z) and scale of later geometry
  s x y z r                                       sphere (centre transformed, radius not)
  p n + n vertex lines "x y z [nx ny nz [u v]]"   polygon, fan-triangulated; flat normals if
                                                  any vertex has none
  m file                                          mesh file (Wavefront OBJ here)
  include file                                    another NFF file in the same scope
  shader name                                     activate a defined shader
  diffuse name r g b k                            Lambert, reflectance k * rgb
  specularreflective name r g b k                 mirror
  speculartransmissivedielectric name ior         glass
  glossy name r g b k alpha                       Beckmann microfacet with alpha
  medium name [s a | sr sg sb ar ag ab] [+ "pf rayleigh" | "pf henleygreenstein g"]
                                                  homogeneous medium (or activate one);
                                                  priority = number of media defined before
  vacuummedium name                               no medium
  simpleatmosphere name cx cy cz r                exponential atmosphere (tabulated here)
  tabulatedatmosphere name cx cy cz r file.json   atmosphere from the reference's table file
  larea name uniform r g b power | larea name     uniform area emitter (or activate one;
                                                  `larea none` deactivates)
  l x y z [r g b k]                               point light
  lsun dx dy dz power [half angle in degrees]     sun (default 0.26)
  lddirection dx dy dz r g b                      distant directional light
  lddome ux uy uz r g b                           dome light
  lenv ux uy uz file                              environment map (PFM, or any format Pillow reads)
Geometry takes the material made of the active shader, medium (the medium inside the
surface) and area emitter; the shader `invisible` makes the surface a pure medium boundary.
Not supported here (an error names them): texture lines, `speculardensedielectric`,
`parallel` area emitters and `yaml{ ... }yaml` sections; the tracer has no counterpart.
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass, field, replace
from pathlib import Path
from typing import Dict, Optional

import numpy as np

from . import abi
from .scene import (AtmosphereSpec, CameraSpec, MaterialSpec, MediumSpec, Scene, directional_light, dome_light,
                    env_map, sun_light)
from .spectral import rgb_to_spectrum

NBINS = abi.NBINS


class NFFError(ValueError):
    pass


@dataclass
class _Shader:
    kind: int
    reflectance: np.ndarray
    alpha: float = 0.0
    ior: float = 1.5
    invisible: bool = False


@dataclass
class _Scope:
    transform: np.ndarray = field(default_factory=lambda: np.eye(4))
    shaders: Dict[str, Optional[_Shader]] = field(default_factory=dict)
    media: Dict[str, int] = field(default_factory=dict)          # name -> scene medium index (-1 vacuum)
    emitters: Dict[str, Optional[np.ndarray]] = field(default_factory=dict)
    named: Dict[str, tuple] = field(default_factory=dict)          # material name -> (shader, medium, emitter)
    shader: str = "default"
    medium: str = "default"
    emitter: str = "none"

    def child(self) -> "_Scope":
        return replace(self, transform=self.transform.copy(), shaders=dict(self.shaders), media=dict(self.media),
                       emitters=dict(self.emitters), named=dict(self.named))


def _default_scope() -> _Scope:
    # AddDefaultMaterials (parse_common.cxx:14-24) with the Scene's shaders (scene.cxx:10-30).
    s = _Scope()
    s.shaders = {"default": _Shader(abi.SHADER_DIFFUSE, rgb_to_spectrum((0.8, 0.8, 0.8))),
                 "black": _Shader(abi.SHADER_DIFFUSE, np.zeros(NBINS)),
                 "invisible": _Shader(abi.SHADER_DIFFUSE, np.zeros(NBINS), invisible=True),
                 "none": None}
    s.media = {"default": -1}
    s.emitters = {"none": None}
    return s


def _rot(axis, a):
    c, s = math.cos(a), math.sin(a)
    m = np.eye(4)
    i, j = {0: (1, 2), 1: (2, 0), 2: (0, 1)}[axis]
    m[i, i], m[i, j], m[j, i], m[j, j] = c, -s, s, c
    return m


def _transform(args):
    n = len(args)
    if n not in (0, 3, 6, 9):
        raise NFFError("bad number of arguments to transform")
    m = np.eye(4)
    if n >= 3:
        m[:3, 3] = args[:3]
    if n >= 6:
        # Heading about y, pitch about x, bank about z (y up, z forward).
        m = m @ _rot(1, args[3]) @ _rot(0, args[4]) @ _rot(2, args[5])
    if n >= 9:
        m = m @ np.diag([args[6], args[7], args[8], 1.0])
    return m


def _floats(tokens, what):
    try:
        return [float(t) for t in tokens]
    except ValueError:
        raise NFFError(f"{what}: expected numbers, got {' '.join(tokens)}") from None


def load_obj(path: Path):
    """Wavefront OBJ: vertices, optional normals, polygons fan-triangulated (negative
    indices allowed), `usemtl` names per triangle.  Returns (vertices, normals or None,
    triangles, material name per triangle)."""
    verts, norms, tris, tri_norms, names = [], [], [], [], []
    current = None
    for raw in Path(path).read_text().splitlines():
        t = raw.split()
        if not t or t[0].startswith("#"):
            continue
        if t[0] == "v":
            verts.append([float(x) for x in t[1:4]])
        elif t[0] == "vn":
            norms.append([float(x) for x in t[1:4]])
        elif t[0] == "usemtl":
            current = t[1] if len(t) > 1 else None
        elif t[0] == "f":
            idx = []
            for c in t[1:]:
                parts = c.split("/")
                vi = int(parts[0])
                ni = int(parts[2]) if len(parts) > 2 and parts[2] else 0
                idx.append((vi - 1 if vi > 0 else len(verts) + vi, (ni - 1 if ni > 0 else len(norms) + ni) if ni else -1))
            for k in range(1, len(idx) - 1):
                tri = (idx[0], idx[k], idx[k + 1])
                tris.append([p[0] for p in tri])
                tri_norms.append([p[1] for p in tri])
                names.append(current)
    v = np.array(verts, np.float64).reshape(-1, 3)
    t = np.array(tris, np.int64).reshape(-1, 3)
    tn = np.array(tri_norms, np.int64).reshape(-1, 3)
    if len(norms) and np.all(tn >= 0):
        # Unshare vertices so that every corner carries its own normal.
        n = np.array(norms, np.float64)
        return v[t.reshape(-1)], n[tn.reshape(-1)], np.arange(3 * len(t)).reshape(-1, 3), names
    return v, None, t, names


class _Parser:
    def __init__(self, scene: Scene, width: Optional[int], height: Optional[int]):
        self.scene = scene
        self.width, self.height = width, height
        self.materials: Dict[tuple, int] = {}
        self.meshes = []  # (vertices, normals or None, triangles, material), added at the end

    # The material of the active things (MakeMaterialFromActiveThings, parsenff.cxx:35-38).
    def material(self, scope: _Scope, shader_name: Optional[str] = None) -> int:
        sname = shader_name if shader_name is not None else scope.shader
        medium = scope.media[scope.medium]
        key = (sname, id(scope.shaders.get(sname)), medium, scope.emitter, id(scope.emitters.get(scope.emitter)))
        if key in self.materials:
            return self.materials[key]
        sh = scope.shaders.get(sname)
        em = scope.emitters.get(scope.emitter)
        if sh is None or sh.invisible:
            m = MaterialSpec(shader=abi.SHADER_DIFFUSE, reflectance=np.zeros(NBINS), medium_inside=medium,
                             volume_boundary=em is None)
        else:
            m = MaterialSpec(shader=sh.kind, reflectance=sh.reflectance.copy(), alpha=sh.alpha, ior_ratio=sh.ior,
                             medium_inside=medium)
        if em is not None:
            m.emission = em.copy()
        idx = self.scene.add_material(m)
        self.materials[key] = idx
        return idx

    def parse(self, lines, scope: _Scope, base: Path, start=0):
        i = start
        while i < len(lines):
            line = lines[i].strip()
            i += 1
            if not line or line.startswith("#"):
                continue
            tok = line.split()
            d, args = tok[0], tok[1:]
            where = f"{base}:{i}: {d}"
            if d == "{":
                i = self.parse(lines, scope.child(), base, i)
                continue
            if d == "}":
                return i
            if d == "yaml{":
                block = []
                while i < len(lines) and not lines[i].startswith("}yaml"):
                    block.append(lines[i])
                    i += 1
                if i >= len(lines):
                    raise NFFError(f"{where}: yaml section not terminated with }}yaml")
                i += 1
                self.yaml_section("\n".join(block), scope, where)
                continue
            if d == "diffusetexture" or d == "exponenttexture":
                raise NFFError(f"{where}: textures are not supported by this reader")
            if d == "transform":
                scope.transform = _transform(_floats(args, where))
            elif d in ("v", "vfisheye"):
                cam = {}
                keys = ["from", "at", "up", "resolution"] + (["angle"] if d == "v" else [])
                for k in keys:
                    while i < len(lines) and (not lines[i].strip() or lines[i].strip().startswith("#")):
                        i += 1
                    t = lines[i].split()
                    i += 1
                    if not t or t[0] != k:
                        raise NFFError(f"{where}: expected '{k}'")
                    cam[k] = _floats(t[1:], where)
                pos, at, up = (np.array(cam[k][:3]) for k in ("from", "at", "up"))
                xres = self.width or int(cam["resolution"][0])
                yres = self.height or int(cam["resolution"][1])
                self.scene.camera = CameraSpec(kind=abi.CAMERA_PINHOLE if d == "v" else abi.CAMERA_FISHEYE,
                                               pos=tuple(pos), dir=tuple(at - pos), up=tuple(up),
                                               fov_deg=cam["angle"][0] if d == "v" else 90.0, xres=xres, yres=yres)
            elif d == "s":
                x, y, z, r = _floats(args[:4], where)
                c = scope.transform @ np.array([x, y, z, 1.0])
                self.scene.add_sphere(c[:3], r, self.material(scope))
            elif d == "p":
                n = int(args[0])
                if n < 3:
                    raise NFFError(f"{where}: a polygon needs at least 3 vertices")
                vs, ns, flat = [], [], False
                for _ in range(n):
                    if i >= len(lines):
                        raise NFFError(f"{where}: missing polygon vertices")
                    f = _floats(lines[i].split(), where)
                    i += 1
                    if len(f) < 3:
                        raise NFFError(f"{where}: bad vertex")
                    vs.append(f[:3])
                    flat |= len(f) < 6
                    ns.append(f[3:6] if len(f) >= 6 else [0.0, 0.0, 0.0])
                self.add_mesh(np.array(vs), None if flat else np.array(ns),
                              np.array([[0, k, k + 1] for k in range(1, n - 1)]), scope, self.material(scope))
            elif d == "m":
                path = base.parent / args[0]
                if path.suffix.lower() != ".obj":
                    raise NFFError(f"{where}: only OBJ mesh files are read here ({path.name})")
                v, nrm, t, names = load_obj(path)
                mats = [self.mesh_material(scope, nm) for nm in names]
                for mid in sorted(set(mats)):
                    sel = np.array([m == mid for m in mats])
                    self.add_mesh(v, nrm, t[sel], scope, mid)
            elif d == "include":
                path = base.parent / args[0]
                self.parse(path.read_text().splitlines(), scope, path)
            elif d == "shader":
                if args[0] not in scope.shaders:
                    raise NFFError(f"{where}: unknown shader {args[0]}")
                scope.shader = args[0]
            elif d == "diffuse":
                r, g, b, k = _floats(args[1:5], where)
                scope.shaders[args[0]] = _Shader(abi.SHADER_DIFFUSE, rgb_to_spectrum((k * r, k * g, k * b)))
                scope.shader = args[0]
            elif d == "specularreflective":
                r, g, b, k = _floats(args[1:5], where)
                scope.shaders[args[0]] = _Shader(abi.SHADER_SPECULAR_REFLECTIVE, rgb_to_spectrum((k * r, k * g, k * b)))
                scope.shader = args[0]
            elif d == "speculartransmissivedielectric":
                scope.shaders[args[0]] = _Shader(abi.SHADER_SPECULAR_DIELECTRIC, np.zeros(NBINS),
                                                 ior=_floats(args[1:2], where)[0])
                scope.shader = args[0]
            elif d == "glossy":
                r, g, b, k, alpha = _floats(args[1:6], where)
                scope.shaders[args[0]] = _Shader(abi.SHADER_MICROFACET, rgb_to_spectrum((k * r, k * g, k * b)),
                                                 alpha=alpha)
                scope.shader = args[0]
            elif d == "medium":
                if len(args) == 1:
                    self.activate(scope.media, args[0], where)
                    scope.medium = args[0]
                    continue
                vals = _floats(args[1:], where)
                if len(vals) == 2:
                    ss, sa = rgb_to_spectrum((vals[0],) * 3), rgb_to_spectrum((vals[1],) * 3)
                elif len(vals) == 6:
                    ss, sa = rgb_to_spectrum(vals[0:3]), rgb_to_spectrum(vals[3:6])
                else:
                    raise NFFError(f"{where}: bad medium")
                phase, g = abi.PHASE_UNIFORM, 0.0
                if i < len(lines) and lines[i].strip().startswith("pf "):
                    pf = lines[i].split()
                    i += 1
                    if pf[1] == "rayleigh":
                        phase = abi.PHASE_RAYLEIGH
                    elif pf[1] == "henleygreenstein" and len(pf) > 2:
                        phase, g = abi.PHASE_HENYEY_GREENSTEIN, float(pf[2])
                    else:
                        raise NFFError(f"{where}: bad phase function")
                med = self.scene.add_medium(MediumSpec(sigma_s=np.maximum(ss, 0), sigma_a=np.maximum(sa, 0),
                                                       phase=phase, phase_g=g, priority=len(scope.media)))
                scope.media[args[0]] = med
                scope.medium = args[0]
            elif d == "vacuummedium":
                scope.media[args[0]] = -1
                scope.medium = args[0]
            elif d in ("simpleatmosphere", "tabulatedatmosphere"):
                if len(args) == 1:
                    self.activate(scope.media, args[0], where)
                    scope.medium = args[0]
                    continue
                cx, cy, cz, rad = _floats(args[1:5], where)
                if d == "simpleatmosphere":
                    from .scenes import simple_atmosphere_table
                    h0, dh = -1.0, 0.05
                    tab = simple_atmosphere_table(h0, dh)
                else:
                    data = json.loads((base.parent / args[5]).read_text())
                    h0, dh = float(data["H0"]), float(data["deltaH"])
                    tab = (np.array(data["sigma_t"]), np.array(data["sigma_s_molecules"]),
                           np.array(data["sigma_s_aerosoles"]))
                med = self.scene.add_medium(AtmosphereSpec(planet_center=(cx, cy, cz), planet_radius=rad, h0=h0,
                                                           dh=dh, sigma_t=tab[0], sigma_s_molecules=tab[1],
                                                           sigma_s_aerosols=tab[2], priority=len(scope.media)))
                scope.media[args[0]] = med
                scope.medium = args[0]
            elif d == "larea":
                if len(args) == 1:
                    self.activate(scope.emitters, args[0], where)
                    scope.emitter = args[0]
                    continue
                if args[1] != "uniform":
                    raise NFFError(f"{where}: only uniform area emitters are supported")
                r, g, b, power = _floats(args[2:6], where)
                scope.emitters[args[0]] = power * rgb_to_spectrum((r, g, b))
                scope.emitter = args[0]
            elif d == "l":
                v = _floats(args, where)
                if len(v) == 3:
                    spec = rgb_to_spectrum((1.0, 1.0, 1.0))
                elif len(v) == 7:
                    spec = rgb_to_spectrum((v[6] * v[3], v[6] * v[4], v[6] * v[5]))
                else:
                    raise NFFError(f"{where}: bad point light")
                self.scene.add_point_light(spec, tuple(v[:3]))
            elif d == "lsun":
                v = _floats(args, where)
                dvec = np.array(v[:3]) / np.linalg.norm(v[:3])
                self.scene.env_lights.append(sun_light(v[3], tuple(dvec), v[4] if len(v) > 4 else 0.26))
            elif d == "lddirection":
                v = _floats(args, where)
                dvec = np.array(v[:3]) / np.linalg.norm(v[:3])
                self.scene.env_lights.append(directional_light(rgb_to_spectrum(v[3:6]), tuple(dvec)))
            elif d == "lddome":
                v = _floats(args, where)
                up = np.array(v[:3]) / np.linalg.norm(v[:3])
                self.scene.env_lights.append(dome_light(rgb_to_spectrum(v[3:6]), tuple(up)))
            elif d == "lenv":
                v = _floats(args[:3], where)
                self.scene.env_lights.append(env_map(read_image(base.parent / args[3]), tuple(v)))
            else:
                raise NFFError(f"{where}: unknown directive")
        return i

    def yaml_section(self, text: str, scope: _Scope, where: str):
        """NFFParser::ParseYamlNode (parsenff.cxx:868-970): transform (replaces the current
        one; radians unless angle_in_degree), shader (speculartransmissivedielectric or glossy
        with rgb and x; activated), material (names the active shader, medium and emitter)."""
        import yaml
        doc = yaml.safe_load(text) or {}
        for key, node in doc.items():
            if key == "transform":
                f = math.pi / 180.0 if node.get("angle_in_degree") else 1.0
                m = np.eye(4)
                if "pos" in node:
                    m[:3, 3] = [float(x) for x in node["pos"]]
                if "hpb" in node:
                    h, p, b = (float(x) * f for x in node["hpb"])
                    m = m @ _rot(1, h) @ _rot(0, p) @ _rot(2, b)
                if "rotaxis" in node:
                    from .yaml_scene import _axis_angle
                    r = np.array([float(x) for x in node["rotaxis"]]) * f
                    n = np.linalg.norm(r)
                    if n > 0:
                        m = m @ _axis_angle(r / n, n)
                if "scale" in node:
                    m = m @ np.diag([float(x) for x in node["scale"]] + [1.0])
                scope.transform = m
            elif key == "shader":
                cls, name = node["class"], node["name"]
                if cls == "speculartransmissivedielectric":
                    if "abbe_number" in node:
                        raise NFFError(f"{where}: dispersion (abbe_number) is not supported")
                    scope.shaders[name] = _Shader(abi.SHADER_SPECULAR_DIELECTRIC, np.zeros(NBINS),
                                                  ior=float(node["ior_ratio"]))
                elif cls == "glossytransmissivedielectric":
                    if "alpha_texture" in node:
                        raise NFFError(f"{where}: roughness textures are not supported")
                    scope.shaders[name] = _Shader(abi.SHADER_GLOSSY_DIELECTRIC, np.zeros(NBINS),
                                                  ior=float(node["ior_ratio"]), alpha=float(node["alpha"]))
                elif cls == "glossy":
                    rgb = [float(x) for x in node.get("rgb", [1.0, 1.0, 1.0])]
                    k = float(node.get("x", 1.0))
                    scope.shaders[name] = _Shader(abi.SHADER_MICROFACET, rgb_to_spectrum([k * x for x in rgb]),
                                                  alpha=float(node["alpha"]))
                else:
                    raise NFFError(f"{where}: shader class {cls} is not supported by this tracer")
                scope.shader = name
            elif key == "material":
                scope.named[node["name"]] = (scope.shader, scope.medium, scope.emitter)
            else:
                raise NFFError(f"{where}: yaml key {key} is not supported")

    @staticmethod
    def activate(table, name, where):
        if name not in table:
            raise NFFError(f"{where}: {name} is not defined")

    def mesh_material(self, scope: _Scope, name: Optional[str]) -> int:
        # GetMaterial (parsenff.cxx:41-66): a defined shader of that name, else the active material.
        if name and name != "DefaultMaterial":
            if name in scope.named:
                s = scope.child()
                s.shader, s.medium, s.emitter = scope.named[name]
                return self.material(s)
            if name in scope.shaders:
                return self.material(scope, name)
        return self.material(scope)

    def add_mesh(self, v, n, t, scope: _Scope, material: int):
        M = scope.transform
        vh = np.c_[v, np.ones(len(v))] @ M.T
        nn = None
        if n is not None:
            N = np.linalg.inv(M[:3, :3]).T
            nn = n @ N.T
            nn /= np.maximum(np.linalg.norm(nn, axis=1, keepdims=True), 1e-30)
        used = np.unique(t)
        remap = -np.ones(len(v), np.int64)
        remap[used] = np.arange(len(used))
        self.meshes.append((vh[used, :3], None if nn is None else nn[used], remap[t], material))

    def finish(self):
        # The Scene carries normals for all meshes or for none: meshes without get flat ones
        # (Mesh::MakeFlatNormals: every triangle its own vertices and geometric normal).
        any_n = any(n is not None for _, n, _, _ in self.meshes)
        for v, n, t, m in self.meshes:
            if any_n and n is None:
                v = v[t.reshape(-1)]
                t = np.arange(len(v)).reshape(-1, 3)
                g = np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
                g /= np.maximum(np.linalg.norm(g, axis=1, keepdims=True), 1e-30)
                n = np.repeat(g, 3, axis=0)
            self.scene.add_mesh(v, t, m, n)


def read_image(path: Path) -> np.ndarray:
    """Float RGB image, row 0 at the top: PFM read here, other formats through Pillow."""
    path = Path(path)
    if path.suffix.lower() == ".pfm":
        return read_pfm(path)
    try:
        from PIL import Image
    except ImportError:
        raise NFFError(f"cannot read {path.name}: only PFM is read without Pillow") from None
    return np.asarray(Image.open(path).convert("RGB"), np.float32) / 255.0


def read_pfm(path: Path) -> np.ndarray:
    """Portable float map: 'PF' header (RGB), width height, scale (< 0: little endian), rows
    from the bottom."""
    data = Path(path).read_bytes()
    parts = data.split(b"\n", 3)
    if parts[0].strip() != b"PF":
        raise NFFError(f"{path}: not an RGB PFM file")
    w, h = (int(x) for x in parts[1].split())
    scale = float(parts[2])
    img = np.frombuffer(parts[3], dtype="<f4" if scale < 0 else ">f4", count=w * h * 3).reshape(h, w, 3)
    return np.ascontiguousarray(img[::-1], dtype=np.float32)


def parse_nff(source, width: Optional[int] = None, height: Optional[int] = None) -> Scene:
    """Scene from an NFF file path or text (Scene::ParseNFF, parsenff.cxx:982-996).
    width / height override the file's resolution, as RenderingParameters do."""
    scene = Scene()
    p = Path(source) if not isinstance(source, str) or "\n" not in source else None
    if p is not None and p.exists():
        text, base = p.read_text(), p
        scene.name = p.stem
    else:
        text, base = str(source), Path("scene.nff")
        scene.name = "nff"
    parser = _Parser(scene, width, height)
    parser.parse(text.splitlines(), _default_scope(), base.resolve() if p is not None else base)
    parser.finish()
    return scene
