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
  m file                                          mesh file (Wavefront OBJ or COLLADA .dae)
  include file                                    another NFF file in the same scope
  shader name                                     activate a defined shader
  diffuse name r g b k [+ "diffusetexture file"]  Lambert, reflectance k * rgb (times the
                                                  texture's linear RGB at the hit)
  specularreflective name r g b k                 mirror
  speculardensedielectric name r g b k [+ texture] smooth coating (reflectivity k) over Lambert rgb
  speculartransmissivedielectric name ior         glass
  glossy name r g b k alpha                       Beckmann microfacet with alpha
  medium name [s a | sr sg sb ar ag ab] [+ "pf rayleigh" | "pf henleygreenstein g"]
                                                  homogeneous medium (or activate one);
                                                  priority = number of media defined before
  vacuummedium name                               no medium
  simpleatmosphere name cx cy cz r                exponential atmosphere (tabulated here)
  tabulatedatmosphere name cx cy cz r file.json   atmosphere from the reference's table file
  larea name uniform|parallel r g b power        uniform or parallel area emitter, or
  larea name                                      activate one (`larea none` deactivates)
  l x y z [r g b k]                               point light
  lsun dx dy dz power [half angle in degrees]     sun (default 0.26)
  lddirection dx dy dz r g b                      distant directional light
  lddome ux uy uz r g b                           dome light
  lenv ux uy uz file                              environment map (PFM, or any format Pillow reads)
Geometry takes the material made of the active shader, medium (the medium inside the
surface) and area emitter; the shader `invisible` makes the surface a pure medium boundary.
Not supported here (an error names them): roughness textures and the yaml keys the tracer
has no counterpart for.
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
    texture: int = -1  # scene texture multiplying the diffuse reflectance
    specular: float = 0.0  # dense dielectric coating reflectivity


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


def _axis_angle(axis, angle):
    """Rotation by `angle` (radians) about the unit vector `axis`, as a 4x4 matrix."""
    x, y, z = axis
    c, s, t = math.cos(angle), math.sin(angle), 1 - math.cos(angle)
    m = np.eye(4)
    m[:3, :3] = [[t * x * x + c, t * x * y - s * z, t * x * z + s * y],
                 [t * x * y + s * z, t * y * y + c, t * y * z - s * x],
                 [t * x * z - s * y, t * y * z + s * x, t * z * z + c]]
    return m


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
    """Wavefront OBJ: vertices, optional texture coordinates and normals, polygons
    fan-triangulated (negative indices allowed), `usemtl` names per triangle.  When faces
    carry normals or texture coordinates every triangle corner gets its own vertex (as the
    reference's assimp import makes them).  Returns (vertices, normals or None, triangles,
    material name per triangle, texture coordinates or None)."""
    verts, uvs, norms, tris, names = [], [], [], [], []
    current = None

    def ref(s, n):
        if not s:
            return -1
        k = int(s)
        return k - 1 if k > 0 else n + k

    for raw in Path(path).read_text().splitlines():
        t = raw.split()
        if not t or t[0].startswith("#"):
            continue
        if t[0] == "v":
            verts.append([float(x) for x in t[1:4]])
        elif t[0] == "vt":
            uvs.append([float(x) for x in t[1:3]] + [0.0] * max(0, 3 - len(t)))
        elif t[0] == "vn":
            norms.append([float(x) for x in t[1:4]])
        elif t[0] == "usemtl":
            current = t[1] if len(t) > 1 else None
        elif t[0] == "f":
            idx = []
            for c in t[1:]:
                parts = c.split("/") + ["", ""]
                idx.append((ref(parts[0], len(verts)), ref(parts[1], len(uvs)), ref(parts[2], len(norms))))
            for k in range(1, len(idx) - 1):
                tris.append((idx[0], idx[k], idx[k + 1]))
                names.append(current)
    v = np.array(verts, np.float64).reshape(-1, 3)
    c = np.array(tris, np.int64).reshape(-1, 3, 3)  # triangle, corner, (v, vt, vn)
    t = c[:, :, 0]
    has_n = len(norms) > 0 and len(c) > 0 and bool(np.all(c[:, :, 2] >= 0))
    has_uv = len(uvs) > 0 and len(c) > 0 and bool(np.all(c[:, :, 1] >= 0))
    if not (has_n or has_uv):
        return v, None, t, names, None
    # Unshare vertices so that every corner carries its own normal and coordinates.
    n = np.array(norms, np.float64)[c[:, :, 2].reshape(-1)] if has_n else None
    uv = np.array(uvs, np.float64)[c[:, :, 1].reshape(-1)][:, :2] if has_uv else None
    return v[t.reshape(-1)], n, np.arange(3 * len(t)).reshape(-1, 3), names, uv


def _dae_floats(text):
    return [float(x) for x in (text or "").split()]


def _dae_node_matrix(node, ns):
    """Local transform of a COLLADA <node>: its transform elements composed in document
    order (translate, rotate axis+degrees, scale, matrix)."""
    M = np.eye(4)
    for el in node:
        tag = el.tag[len(ns):]
        v = _dae_floats(el.text)
        if tag == "translate":
            T = np.eye(4)
            T[:3, 3] = v[:3]
        elif tag == "rotate":
            ax = np.array(v[:3], np.float64)
            n = np.linalg.norm(ax)
            T = np.eye(4)
            if n > 0:
                T[:3, :3] = _axis_angle(ax / n, math.radians(v[3]))[:3, :3]
        elif tag == "scale":
            T = np.diag(v[:3] + [1.0])
        elif tag == "matrix":
            T = np.array(v[:16], np.float64).reshape(4, 4)
        else:
            continue
        M = M @ T
    return M


def load_dae(path: Path):
    """COLLADA (.dae) triangle meshes, as the reference's assimp import delivers them for
    the `m` directive (scenereader::assimp::Read, parse_common.cxx:106-239): every
    <instance_geometry> of the visual scene's node tree with the node transforms composed
    from the root, positions scaled by the asset's <unit meter>, <triangles> and <polylist>
    (fan-triangulated) faces with one vertex per face corner, normals when the mesh has them,
    faces of zero area dropped (CheckFace), and per face the name of the material bound to
    its material symbol.  Only Y_UP assets are read.  Returns (vertices, normals or None,
    triangles, material name per triangle, texture coordinates or None)."""
    import xml.etree.ElementTree as ET
    root = ET.parse(path).getroot()
    ns = root.tag[: root.tag.index("}") + 1] if root.tag.startswith("{") else ""
    q = lambda tag: ns + tag  # noqa: E731
    unit = root.find(f"{q('asset')}/{q('unit')}")
    scale = float(unit.get("meter", "1")) if unit is not None else 1.0
    up = root.find(f"{q('asset')}/{q('up_axis')}")
    if up is not None and (up.text or "").strip() not in ("Y_UP", ""):
        raise ValueError(f"up axis {up.text.strip()} (only Y_UP is read)")
    mat_names = {m.get("id"): m.get("name", m.get("id")) for m in root.iter(q("material"))}
    geoms = {g.get("id"): g for g in root.iter(q("geometry"))}
    verts, norms, uvs, names = [], [], [], []
    has_normals = True
    has_uvs = True

    def mesh_faces(geom, M, binding):
        nonlocal has_normals, has_uvs
        mesh = geom.find(q("mesh"))
        if mesh is None:
            return
        sources = {}
        for src in mesh.findall(q("source")):
            arr = src.find(q("float_array"))
            acc = src.find(f"{q('technique_common')}/{q('accessor')}")
            stride = int(acc.get("stride", "1")) if acc is not None else 1
            vals = np.array(_dae_floats(arr.text if arr is not None else ""), np.float64)
            sources["#" + src.get("id")] = vals.reshape(-1, stride)
        vinput = mesh.find(q("vertices"))
        vsrc = {i.get("semantic"): i.get("source") for i in vinput.findall(q("input"))} if vinput is not None else {}
        N = np.linalg.inv(M[:3, :3]).T
        for prim in list(mesh.findall(q("triangles"))) + list(mesh.findall(q("polylist"))):
            inputs = prim.findall(q("input"))
            stride = max(int(i.get("offset", "0")) for i in inputs) + 1
            idx = np.array([int(x) for x in (prim.find(q("p")).text or "").split()], np.int64).reshape(-1, stride)
            if prim.tag == q("polylist"):
                counts = [int(x) for x in prim.find(q("vcount")).text.split()]
            else:
                counts = [3] * (len(idx) // 3)
            pos = nrm = tc = None
            for inp in inputs:
                sem, off = inp.get("semantic"), int(inp.get("offset", "0"))
                if sem == "VERTEX":
                    pos = sources[vsrc["POSITION"]][idx[:, off]][:, :3]
                    if "NORMAL" in vsrc:
                        nrm = sources[vsrc["NORMAL"]][idx[:, off]][:, :3]
                    if "TEXCOORD" in vsrc:
                        tc = sources[vsrc["TEXCOORD"]][idx[:, off]][:, :2]
                elif sem == "NORMAL":
                    nrm = sources[inp.get("source")][idx[:, off]][:, :3]
                elif sem == "TEXCOORD" and inp.get("set", "0") == "0" and tc is None:
                    tc = sources[inp.get("source")][idx[:, off]][:, :2]
            if pos is None:
                raise ValueError("a face set without positions")
            pw = np.c_[pos, np.ones(len(pos))] @ M.T
            name = mat_names.get(binding.get(prim.get("material")), prim.get("material"))
            start = 0
            for cnt in counts:
                for k in range(1, cnt - 1):
                    c = [start, start + k, start + k + 1]
                    tri = pw[c, :3] * scale
                    if np.linalg.norm(np.cross(tri[1] - tri[0], tri[2] - tri[0])) > 0.0:
                        verts.append(tri)
                        if nrm is not None:
                            nn = nrm[c] @ N.T
                            norms.append(nn / np.maximum(np.linalg.norm(nn, axis=1, keepdims=True), 1e-30))
                        else:
                            has_normals = False
                        if tc is not None and tc.shape[1] >= 2:
                            uvs.append(tc[c, :2])
                        else:
                            has_uvs = False
                        names.append(name)
                start += cnt

    def walk(node, parent):
        M = parent @ _dae_node_matrix(node, ns)
        for ig in node.findall(q("instance_geometry")):
            binding = {im.get("symbol"): (im.get("target") or "").lstrip("#")
                       for im in ig.iter(q("instance_material"))}
            geom = geoms.get((ig.get("url") or "").lstrip("#"))
            if geom is None:
                raise ValueError(f"geometry {ig.get('url')} not found")
            mesh_faces(geom, M, binding)
        for child in node.findall(q("node")):
            walk(child, M)

    scene_ref = root.find(f"{q('scene')}/{q('instance_visual_scene')}")
    vscenes = {v.get("id"): v for v in root.iter(q("visual_scene"))}
    vs = vscenes.get((scene_ref.get("url") or "").lstrip("#")) if scene_ref is not None else None
    if vs is None and vscenes:
        vs = next(iter(vscenes.values()))
    if vs is None:
        raise ValueError("no visual scene")
    for node in vs.findall(q("node")):
        walk(node, np.eye(4))
    if not verts:
        raise ValueError("no triangles")
    v = np.concatenate(verts)
    t = np.arange(len(v)).reshape(-1, 3)
    n = np.concatenate(norms) if has_normals and norms else None
    uv = np.concatenate(uvs) if has_uvs and uvs else None
    return v, n, t, names, uv


class _Parser:
    def __init__(self, scene: Scene, width: Optional[int], height: Optional[int]):
        self.scene = scene
        self.width, self.height = width, height
        self.materials: Dict[tuple, int] = {}
        self.meshes = []  # (vertices, normals or None, triangles, material, uvs or None), added at the end
        self.textures: Dict[str, int] = {}  # image file -> scene texture index

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
                             medium_inside=medium, diffuse_texture=sh.texture, specular_reflectivity=sh.specular)
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
                raise NFFError(f"{where}: {d}: only a diffusetexture right after a diffuse shader is read")
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
                vs, ns, us, flat, no_uv = [], [], [], False, False
                for _ in range(n):
                    if i >= len(lines):
                        raise NFFError(f"{where}: missing polygon vertices")
                    f = _floats(lines[i].split(), where)
                    i += 1
                    if len(f) < 3:
                        raise NFFError(f"{where}: bad vertex")
                    vs.append(f[:3])
                    flat |= len(f) < 6
                    no_uv |= len(f) < 8
                    ns.append(f[3:6] if len(f) >= 6 else [0.0, 0.0, 0.0])
                    us.append(f[6:8] if len(f) >= 8 else [0.0, 0.0])
                self.add_mesh(np.array(vs), None if flat else np.array(ns),
                              np.array([[0, k, k + 1] for k in range(1, n - 1)]), scope, self.material(scope),
                              None if no_uv else np.array(us))
            elif d == "m":
                path = base.parent / args[0]
                if path.suffix.lower() == ".obj":
                    v, nrm, t, names, uv = load_obj(path)
                elif path.suffix.lower() == ".dae":
                    try:
                        v, nrm, t, names, uv = load_dae(path)
                    except (ValueError, KeyError) as e:
                        raise NFFError(f"{where}: {path.name}: {e}") from e
                else:
                    raise NFFError(f"{where}: mesh format {path.suffix} is not read here (OBJ and COLLADA are)")
                mats = [self.mesh_material(scope, nm) for nm in names]
                for mid in sorted(set(mats)):
                    sel = np.array([m == mid for m in mats])
                    self.add_mesh(v, nrm, t[sel], scope, mid, uv)
            elif d == "include":
                path = base.parent / args[0]
                self.parse(path.read_text().splitlines(), scope, path)
            elif d == "shader":
                if args[0] not in scope.shaders:
                    raise NFFError(f"{where}: unknown shader {args[0]}")
                scope.shader = args[0]
            elif d == "diffuse":
                r, g, b, k = _floats(args[1:5], where)
                tex = -1
                # MaybeReadTexture (parsenff.cxx:350-368): a `diffusetexture file` line right after.
                if i < len(lines) and lines[i].strip().startswith("diffusetexture"):
                    targs = lines[i].split()[1:]
                    i += 1
                    if len(targs) != 1:
                        raise NFFError(f"{base}:{i}: diffusetexture needs a file name")
                    tex = self.texture(base.parent / targs[0])
                scope.shaders[args[0]] = _Shader(abi.SHADER_DIFFUSE, rgb_to_spectrum((k * r, k * g, k * b)),
                                                 texture=tex)
                scope.shader = args[0]
            elif d == "speculardensedielectric":
                # parsenff.cxx:416-431: diffuse rgb (no factor), then the coating's reflectivity.
                r, g, b, k = _floats(args[1:5], where)
                tex = -1
                if i < len(lines) and lines[i].strip().startswith("diffusetexture"):
                    targs = lines[i].split()[1:]
                    i += 1
                    if len(targs) != 1:
                        raise NFFError(f"{base}:{i}: diffusetexture needs a file name")
                    tex = self.texture(base.parent / targs[0])
                scope.shaders[args[0]] = _Shader(abi.SHADER_SPECULAR_DENSE_DIELECTRIC, rgb_to_spectrum((r, g, b)),
                                                 texture=tex, specular=k)
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
                if args[1] not in ("uniform", "parallel"):
                    raise NFFError(f"{where}: area emitter type {args[1]} is unknown")
                r, g, b, power = _floats(args[2:6], where)
                # ParallelAreaLight (light.hxx:112-146) radiates only along the winding normal,
                # a delta direction that a camera path's light sample or scattered ray never
                # meets: under forward path tracing it is a light the picker selects (its
                # triangles count as area lights) that contributes nothing.
                scope.emitters[args[0]] = (power * rgb_to_spectrum((r, g, b)) if args[1] == "uniform"
                                           else np.zeros(NBINS))
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

    def add_mesh(self, v, n, t, scope: _Scope, material: int, uv=None):
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
        self.meshes.append((vh[used, :3], None if nn is None else nn[used], remap[t], material,
                            None if uv is None else np.asarray(uv, np.float64)[used]))

    def texture(self, path: Path) -> int:
        """Scene texture index of an image file (read once per file)."""
        key = str(Path(path).resolve())
        if key not in self.textures:
            self.textures[key] = self.scene.add_texture(read_texture(path))
        return self.textures[key]

    def finish(self):
        # The Scene carries normals for all meshes or for none: meshes without get flat ones
        # (Mesh::MakeFlatNormals: every triangle its own vertices and geometric normal).
        any_n = any(n is not None for _, n, _, _, _ in self.meshes)
        for v, n, t, m, uv in self.meshes:
            if any_n and n is None:
                v = v[t.reshape(-1)]
                if uv is not None:
                    uv = uv[t.reshape(-1)]
                t = np.arange(len(v)).reshape(-1, 3)
                g = np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
                g /= np.maximum(np.linalg.norm(g, axis=1, keepdims=True), 1e-30)
                n = np.repeat(g, 3, axis=0)
            self.scene.add_mesh(v, t, m, n, uv)


def srgb_to_linear(x):
    """Color::SRGBToLinear (spectral.hxx:144-149)."""
    x = np.asarray(x, np.float64)
    return np.where(x <= 0.04045, x / 12.92, ((x + 0.055) / 1.055) ** 2.4)


def read_image(path: Path) -> np.ndarray:
    """Linear float RGB image, row 0 at the top: PFM and OpenEXR as stored, 8-bit formats
    through Pillow with the sRGB curve undone (Texture::GetPixel, texture.hxx:94-117)."""
    path = Path(path)
    if path.suffix.lower() == ".pfm":
        return read_pfm(path)
    if path.suffix.lower() == ".exr":
        from .image import read_exr
        return read_exr(path)
    try:
        from PIL import Image
    except ImportError:
        raise NFFError(f"cannot read {path.name}: only PFM and EXR are read without Pillow") from None
    return srgb_to_linear(np.asarray(Image.open(path).convert("RGB"), np.float64) / 255.0).astype(np.float32)


def read_texture(path: Path) -> np.ndarray:
    return np.ascontiguousarray(read_image(path), dtype=np.float32)


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
