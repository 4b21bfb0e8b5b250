"""Reader for the reference's YAML scene files (YamlSceneReader, src/parse_yaml_scene.cxx)
into a `Scene` for the CUDA tracer.

A file is one scope: a mapping with any of
  transforms: [{pos: [x,y,z]} | {hpb: [h,p,b], rad: bool} | {rotaxis: [x,y,z], rad: bool} |
               {scale: [x,y,z]}, ...]   composed in order onto the scope's transform
               (degrees unless rad: true)
  shaders:    [{name, class: diffuse | glossy | speculartransmissivedielectric |
                glossytransmissivedielectric | speculardensedielectric, rgb, rgb_x, alpha, ior_ratio,
                specular, texture}, ...]
  media:      [{name, class: homogeneous, absorb, absorb_x, scatter, scatter_x,
                phasefunction: {class: rayleigh | henleygreenstein, g}}, ...]
  arealights: [{name, class: uniform | parallel, rgb, rgb_x}, ...]
  lights:     [{class: point, position, rgb, rgb_x} | {class: sun, direction, total_power,
                opening_angle_deg} | {class: directional | dome, direction, rgb, rgb_x} |
               {class: env, direction, filename}, ...]
  materials:  [{name, shader, medium, outer_medium, arealight}, ...]  each a name or an
               inlined item
  models:     [{sphere, position, radius, defaultmaterial} |
               {file: mesh.obj | mesh.dae, defaultmaterial, materialmap: {mesh material: material}}, ...]
  scopes:     [scope, ...]  nested, inheriting and then forgetting definitions and transform
  view:       {from, at, up, angle}  (resolution from the caller, default 640 x 480)
Sections are read in the reference's order (transforms, shaders, media, arealights, lights,
materials, models, scopes, view).  Colours are RGB (default 1) times the `_x` factor,
converted to spectra.  A sphere's radius scales with the cube root of the transform's
determinant.  Classes the tracer has no counterpart for (modulated-density media,
roughness textures) raise an error naming them.
"""
from __future__ import annotations

import math
from dataclasses import replace
from pathlib import Path
from typing import Optional

import numpy as np

from . import abi
from .nff import NFFError, _axis_angle, _Parser, _Scope, _Shader, _default_scope, load_dae, load_obj, read_image
from .scene import CameraSpec, MediumSpec, Scene, directional_light, dome_light, env_map, sun_light
from .spectral import rgb_to_spectrum

NBINS = abi.NBINS


def _spectrum(node: dict, prefix: str) -> np.ndarray:
    rgb = node.pop(prefix, [1.0, 1.0, 1.0])
    k = float(node.pop(prefix + "_x", 1.0))
    return rgb_to_spectrum([k * float(x) for x in rgb])


def parse_transform(items) -> np.ndarray:
    """YamlSceneReader::ParseTransform (parse_yaml_scene.cxx:222-258)."""
    m = np.eye(4)
    for it in items if isinstance(items, list) else [items]:
        it = dict(it)
        rad = bool(it.pop("rad", False))
        f = 1.0 if rad else math.pi / 180.0
        if "pos" in it:
            t = np.eye(4)
            t[:3, 3] = [float(x) for x in it.pop("pos")]
            m = m @ t
        elif "hpb" in it:
            h, p, b = (float(x) * f for x in it.pop("hpb"))
            m = m @ _axis_angle((0, 1, 0), h) @ _axis_angle((1, 0, 0), p) @ _axis_angle((0, 0, 1), b)
        if "rotaxis" in it:
            r = np.array([float(x) for x in it.pop("rotaxis")]) * f
            n = np.linalg.norm(r)
            if n > 0:
                m = m @ _axis_angle(r / n, n)
        if "scale" in it:
            m = m @ np.diag([float(x) for x in it.pop("scale")] + [1.0])
        if it:
            raise NFFError(f"transform: unknown keys {sorted(it)}")
    return m


class _YamlReader(_Parser):
    def __init__(self, scene: Scene, width, height, base: Path):
        super().__init__(scene, width, height)
        self.base = base

    # -- items ------------------------------------------------------------------------
    def shader(self, node: dict, scope: _Scope) -> str:
        node = dict(node)
        name = node.pop("name", None) or f"_inline{len(scope.shaders)}"
        cls = node.pop("class")
        node.pop("prefer_path_tracing", None)
        if cls == "diffuse":
            tex = node.pop("texture", None)
            sh = _Shader(abi.SHADER_DIFFUSE, _spectrum(node, "rgb"),
                         texture=self.texture(self.base.parent / tex) if tex else -1)
        elif cls == "glossy":
            alpha = float(node.pop("alpha"))
            sh = _Shader(abi.SHADER_MICROFACET, _spectrum(node, "rgb"), alpha=alpha)
        elif cls == "speculartransmissivedielectric":
            ior = float(node.pop("ior_ratio"))
            if "abbe_number" in node:
                raise NFFError("shader: dispersion (abbe_number) is not supported")
            sh = _Shader(abi.SHADER_SPECULAR_DIELECTRIC, np.zeros(NBINS), ior=ior)
        elif cls == "speculardensedielectric":
            # parse_yaml_scene.cxx:474-480
            spec = float(node.pop("specular"))
            tex = node.pop("texture", None)
            sh = _Shader(abi.SHADER_SPECULAR_DENSE_DIELECTRIC, _spectrum(node, "rgb"),
                         texture=self.texture(self.base.parent / tex) if tex else -1, specular=spec)
        elif cls == "glossytransmissivedielectric":
            # parse_yaml_scene.cxx:443-450 (alpha_min only with a roughness texture)
            ior = float(node.pop("ior_ratio"))
            alpha = float(node.pop("alpha"))
            if "alpha_texture" in node:
                raise NFFError("shader: roughness textures are not supported")
            sh = _Shader(abi.SHADER_GLOSSY_DIELECTRIC, np.zeros(NBINS), ior=ior, alpha=alpha)
        else:
            raise NFFError(f"shader class {cls} is not supported by this tracer")
        if node:
            raise NFFError(f"shader {name}: unknown keys {sorted(node)}")
        scope.shaders[name] = sh
        return name

    def medium(self, node: dict, scope: _Scope) -> str:
        node = dict(node)
        name = node.pop("name", None) or f"_inline{len(scope.media)}"
        cls = node.pop("class")
        if cls != "homogeneous":
            raise NFFError(f"medium class {cls} is not supported by this tracer")
        absorb, scatter = _spectrum(node, "absorb"), _spectrum(node, "scatter")
        phase, g = abi.PHASE_UNIFORM, 0.0
        pf = node.pop("phasefunction", None)
        if pf is not None:
            pf = dict(pf)
            pc = pf.pop("class")
            if pc == "rayleigh":
                phase = abi.PHASE_RAYLEIGH
            elif pc == "henleygreenstein":
                phase, g = abi.PHASE_HENYEY_GREENSTEIN, float(pf.pop("g", 1.0))
            else:
                raise NFFError(f"phase function {pc} is not supported")
        if node:
            raise NFFError(f"medium {name}: unknown keys {sorted(node)}")
        scope.media[name] = self.scene.add_medium(MediumSpec(sigma_s=np.maximum(scatter, 0),
                                                             sigma_a=np.maximum(absorb, 0), phase=phase,
                                                             phase_g=g, priority=len(scope.media)))
        return name

    def arealight(self, node: dict, scope: _Scope) -> str:
        node = dict(node)
        name = node.pop("name", None) or f"_inline{len(scope.emitters)}"
        cls = node.pop("class")
        if cls not in ("uniform", "parallel"):
            raise NFFError(f"area light class {cls} is unknown")
        spec = _spectrum(node, "rgb")
        # A parallel area light (light.hxx:112-146) emits along the winding normal only: a
        # selected light that contributes nothing to forward path tracing.
        scope.emitters[name] = spec if cls == "uniform" else np.zeros(NBINS)
        if node:
            raise NFFError(f"area light {name}: unknown keys {sorted(node)}")
        return name

    def light(self, node: dict, scope: _Scope):
        node = dict(node)
        cls = node.pop("class")
        if cls == "point":
            spec = _spectrum(node, "rgb")
            pos = scope.transform @ np.array([float(x) for x in node.pop("position")] + [1.0])
            self.scene.add_point_light(spec, tuple(pos[:3]))
        elif cls in ("sun", "directional", "dome", "env"):
            d = np.array([float(x) for x in node.pop("direction")])
            d /= np.linalg.norm(d)
            if cls == "sun":
                power = float(node.pop("total_power"))
                self.scene.env_lights.append(sun_light(power, tuple(-d), float(node.pop("opening_angle_deg", 0.25))))
            elif cls == "directional":
                self.scene.env_lights.append(directional_light(_spectrum(node, "rgb"), tuple(-d)))
            elif cls == "dome":
                self.scene.env_lights.append(dome_light(_spectrum(node, "rgb"), tuple(d)))
            else:
                self.scene.env_lights.append(env_map(read_image(self.base.parent / node.pop("filename")), tuple(d)))
        else:
            raise NFFError(f"light class {cls} is not supported")
        if node:
            raise NFFError(f"light {cls}: unknown keys {sorted(node)}")

    def ref(self, value, kind, scope: _Scope) -> str:
        if isinstance(value, str):
            table = {"shader": scope.shaders, "medium": scope.media, "arealight": scope.emitters}[kind]
            if value not in table:
                raise NFFError(f"unknown {kind} {value}")
            return value
        return {"shader": self.shader, "medium": self.medium, "arealight": self.arealight}[kind](value, scope)

    def material_def(self, node: dict, scope: _Scope, mats: dict):
        node = dict(node)
        name = node.pop("name")
        sh = self.ref(node.pop("shader"), "shader", scope) if "shader" in node else "default"
        med = self.ref(node.pop("medium"), "medium", scope) if "medium" in node else "default"
        outer = self.ref(node.pop("outer_medium"), "medium", scope) if "outer_medium" in node else None
        em = self.ref(node.pop("arealight"), "arealight", scope) if "arealight" in node else "none"
        if node:
            raise NFFError(f"material {name}: unknown keys {sorted(node)}")
        mats[name] = (sh, med, outer, em)

    def material_index(self, scope: _Scope, mats: dict, name: str) -> int:
        if name not in mats:
            raise NFFError(f"unknown material {name}")
        sh, med, outer, em = mats[name]
        s = scope.child()
        s.shader, s.medium, s.emitter = sh, med, em
        idx = self.material(s)
        if outer is not None:
            # A separate material: the cached one has no outer medium.
            m = replace(self.scene.materials[idx], medium_outside=s.media[outer])
            idx = self.scene.add_material(m)
        return idx

    def model(self, node: dict, scope: _Scope, mats: dict):
        node = dict(node)
        default = node.pop("defaultmaterial", "default")
        mmap = dict(node.pop("materialmap", {}) or {})
        node.pop("material_assignment_by_object_names", None)
        if "sphere" in node:
            node.pop("sphere")
            c = scope.transform @ np.array([float(x) for x in node.pop("position")] + [1.0])
            r = float(node.pop("radius")) * abs(np.linalg.det(scope.transform[:3, :3])) ** (1.0 / 3.0)
            self.scene.add_sphere(c[:3], r, self.material_index(scope, mats, default))
        elif "file" in node:
            path = self.base.parent / node.pop("file")
            if path.suffix.lower() == ".obj":
                v, nrm, t, names, uv = load_obj(path)
            elif path.suffix.lower() == ".dae":
                v, nrm, t, names, uv = load_dae(path)
            else:
                raise NFFError(f"model {path.name}: mesh format {path.suffix} is not read here (OBJ and COLLADA are)")
            idx = [self.material_index(scope, mats, mmap.get(nm, default) if nm else default) for nm in names]
            for mid in sorted(set(idx)):
                sel = np.array([i == mid for i in idx])
                self.add_mesh(v, nrm, t[sel], scope, mid, uv)
        else:
            raise NFFError("model needs `sphere` or `file`")
        if node:
            raise NFFError(f"model: unknown keys {sorted(node)}")

    def view(self, node: dict):
        node = dict(node)
        f, a, u = (np.array([float(x) for x in node.pop(k)]) for k in ("from", "at", "up"))
        angle = float(node.pop("angle"))
        if node:
            raise NFFError(f"view: unknown keys {sorted(node)}")
        self.scene.camera = CameraSpec(kind=abi.CAMERA_PINHOLE, pos=tuple(f), dir=tuple(a - f), up=tuple(u),
                                       fov_deg=angle, xres=self.width or 640, yres=self.height or 480)

    def scope(self, node: dict, parent: _Scope, parent_mats: dict):
        # YamlSceneReader::ParseScope (parse_yaml_scene.cxx:103-118).
        scope = parent.child()
        mats = dict(parent_mats)
        node = dict(node or {})
        if "transforms" in node:
            scope.transform = scope.transform @ parse_transform(node.pop("transforms"))
        for item in node.pop("shaders", None) or []:
            self.shader(item, scope)
        for item in node.pop("media", None) or []:
            self.medium(item, scope)
        for item in node.pop("arealights", None) or []:
            self.arealight(item, scope)
        for item in node.pop("lights", None) or []:
            self.light(item, scope)
        for item in node.pop("materials", None) or []:
            self.material_def(item, scope, mats)
        for item in node.pop("models", None) or []:
            self.model(item, scope, mats)
        for item in node.pop("scopes", None) or []:
            self.scope(item, scope, mats)
        if "view" in node:
            self.view(node.pop("view"))
        if node:
            raise NFFError(f"scope: unknown keys {sorted(node)}")


def parse_yaml_scene(source, width: Optional[int] = None, height: Optional[int] = None) -> Scene:
    """Scene from a YAML scene file path or text (Scene::ParseYAML,
    parse_yaml_scene.cxx:622-628)."""
    import yaml
    p = Path(source) if not isinstance(source, str) or "\n" not in source else None
    if p is not None and p.exists():
        text, base = p.read_text(), p.resolve()
    else:
        text, base = str(source), Path("scene.yaml").resolve()
    doc = yaml.safe_load(text) or {}
    scene = Scene()
    scene.name = base.stem
    r = _YamlReader(scene, width, height, base)
    # AddDefaultMaterials (parse_common.cxx:14-24): shaders default / black / invisible,
    # medium default (vacuum), material default.
    r.scope(doc, _default_scope(), {"default": ("default", "default", None, "none")})
    r.finish()
    return scene
