"""The NFF reader (naivetrace_b200/nff.py, following parsenff.cxx:113-831) on scene files
written for these tests (tests/golden/scenes/): camera, transforms and scopes, shaders,
media with phase functions, invisible medium boundaries, area / point / sun / dome lights,
included files, OBJ meshes with per-group shaders; errors name the file and line.  Also the
float image writers (PFM, OpenEXR) round trip."""
from pathlib import Path

import numpy as np
import pytest

from naivetrace_b200 import abi
from naivetrace_b200.image import read_exr, write_exr, write_pfm
from naivetrace_b200.nff import NFFError, parse_nff, read_pfm
from naivetrace_b200.spectral import rgb_to_spectrum

SCENES = Path(__file__).parent / "golden" / "scenes"


def _tris(scene):
    v, n, t, m = scene.arrays()
    return v, n, t, m


def test_room_structure():
    s = parse_nff(SCENES / "room.nff")
    c = s.camera
    assert (c.kind, c.xres, c.yres, c.fov_deg) == (abi.CAMERA_PINHOLE, 40, 30, 45.0)
    np.testing.assert_allclose(c.pos, (0.5, 0.5, -1.5))
    np.testing.assert_allclose(c.dir, (0.0, 0.0, 2.0))
    v, n, t, mat = _tris(s)
    # 3 walls x 2 + panel 1 + box 6 x 2 + light 2 + cube 6 x 2 = 33 triangles; 3 spheres.
    assert len(t) == 33 and s.num_spheres == 3
    kinds = [(m.shader, m.volume_boundary, m.emission is not None) for m in s.materials]
    shaders = {k[0] for k in kinds}
    assert {abi.SHADER_DIFFUSE, abi.SHADER_MICROFACET, abi.SHADER_SPECULAR_REFLECTIVE,
            abi.SHADER_SPECULAR_DIELECTRIC} <= shaders
    # Glossy: alpha 0.2, reflectance 1.0 x rgb.
    gl = [m for m in s.materials if m.shader == abi.SHADER_MICROFACET][0]
    assert gl.alpha == pytest.approx(0.2)
    np.testing.assert_allclose(gl.reflectance, rgb_to_spectrum((0.9, 0.7, 0.4)), rtol=1e-12)
    # Glass sphere with the fog medium inside; the fog is Henyey-Greenstein 0.6.
    glass = [m for m in s.materials if m.shader == abi.SHADER_SPECULAR_DIELECTRIC][0]
    assert glass.ior_ratio == 1.5 and glass.medium_inside == 0
    fog, ink = s.media
    assert fog.phase == abi.PHASE_HENYEY_GREENSTEIN and fog.phase_g == pytest.approx(0.6)
    np.testing.assert_allclose(fog.sigma_s, np.maximum(rgb_to_spectrum((0.5,) * 3), 0))
    assert (fog.priority, ink.priority) == (1, 2)
    np.testing.assert_allclose(ink.sigma_a, np.maximum(rgb_to_spectrum((2, 1, 0.5)), 0))
    box = [m for m in s.materials if m.volume_boundary]
    assert len(box) == 1 and box[0].medium_inside == 1
    # Area light: black shader, emission = power x spectrum of white.
    light = [m for m in s.materials if m.emission is not None]
    assert len(light) == 1
    np.testing.assert_allclose(light[0].emission, 8 * rgb_to_spectrum((1, 1, 1)))
    assert np.all(light[0].reflectance == 0)
    # Point light (0.5 x colour), sun (default half angle 0.26 degrees) and dome.
    assert len(s.point_lights) == 1
    np.testing.assert_allclose(s.point_lights[0][0], rgb_to_spectrum((0.5, 0.45, 0.4)))
    kinds = [e.kind for e in s.env_lights]
    assert kinds == [abi.ENV_SUN, abi.ENV_DOME]
    assert s.env_lights[0].scalar == 5 and s.env_lights[0].scalar2 == pytest.approx(0.26)
    np.testing.assert_allclose(np.linalg.norm(s.env_lights[0].dir), 1.0)


def test_transform_scope_and_obj():
    s = parse_nff(SCENES / "room.nff")
    v, n, t, mat = _tris(s)
    # The glossy panel: heading pi/2 about y maps x to -z, then the translation.
    gl_idx = [i for i, m in enumerate(s.materials) if m.shader == abi.SHADER_MICROFACET][0]
    tri = t[mat == gl_idx][0]
    np.testing.assert_allclose(v[tri], [[0.2, 0.05, 0.6], [0.2, 0.05, 0.3], [0.2, 0.35, 0.6]], atol=1e-6)
    # Explicit normals are rotated too: (0, 1, 0) stays.
    np.testing.assert_allclose(n[tri], [[0, 1, 0]] * 3, atol=1e-6)
    # Spheres after the scope use the outer shaders (grey, then chrome), not the panel's.
    sph, smat = s.sphere_arrays()
    assert s.materials[int(smat[0])].shader == abi.SHADER_DIFFUSE
    assert s.materials[int(smat[1])].shader == abi.SHADER_SPECULAR_REFLECTIVE
    # The OBJ cube: three faces with usemtl grey, three with the active (black) shader.
    cube = np.all(v[t][:, :, 0] >= 0.75 - 1e-6, axis=1) & np.all(v[t][:, :, 2] >= 0.7 - 1e-6, axis=1)
    assert cube.sum() == 12
    refl = np.array([s.materials[m].reflectance.max() for m in mat[cube]])
    assert (refl > 0.5).sum() == 6 and (refl == 0).sum() == 6


def test_resolution_override_and_text_input():
    s = parse_nff(SCENES / "room.nff", width=16, height=12)
    assert (s.camera.xres, s.camera.yres) == (16, 12)
    s2 = parse_nff("vfisheye\nfrom 0 0 0\nat 0 1 0\nup 0 0 1\nresolution 8 8\ns 0 2 0 0.5\n")
    assert s2.camera.kind == abi.CAMERA_FISHEYE and s2.num_spheres == 1


@pytest.mark.parametrize("text,msg", [("v\nfrom 0 0 0\nat 0 0 1\nup 0 1 0\nresolution 4 4\nangle 30\nfoo 1\n", ":7"),
                                      ("yaml{\nlight: 1\n}yaml\n", "not supported"),
                                      ("shader nothere\n", "unknown shader"),
                                      ("larea a spot 1 1 1 1\n", "unknown"),
                                      ("p 2\n0 0 0\n1 0 0\n", "3 vertices")])
def test_errors_name_the_line(text, msg):
    with pytest.raises(NFFError, match=msg):
        parse_nff(text + "\n")


def test_float_image_writers(tmp_path):
    a = np.random.default_rng(0).random(6 * 4 * 3).astype(np.float32)
    write_exr(tmp_path / "a.exr", a, 6, 4)
    np.testing.assert_array_equal(read_exr(tmp_path / "a.exr")[::-1].reshape(-1), a)
    raw = (tmp_path / "a.exr").read_bytes()
    assert raw[:4] == bytes([0x76, 0x2F, 0x31, 0x01]) and raw[4] == 2
    write_pfm(tmp_path / "a.pfm", a, 6, 4)
    np.testing.assert_array_equal(read_pfm(tmp_path / "a.pfm")[::-1].reshape(-1), a)


def test_yaml_scene_structure():
    from naivetrace_b200.yaml_scene import parse_yaml_scene
    s = parse_yaml_scene(SCENES / "room.yaml", width=32, height=24)
    c = s.camera
    assert (c.xres, c.yres, c.fov_deg) == (32, 24, 45.0)
    sph, smat = s.sphere_arrays()
    assert len(sph) == 3
    # Scaled scope: radius x cube root of det(0.5^3) = 0.05; centre translated.
    np.testing.assert_allclose(sph[1], [0.5, 0.98, 0.5, 0.05], atol=1e-6)
    np.testing.assert_allclose(sph[2], [0.2, 0.2, 0.3, 0.12], atol=1e-6)
    glass = s.materials[int(smat[0])]
    assert glass.shader == abi.SHADER_SPECULAR_DIELECTRIC and glass.ior_ratio == pytest.approx(1.33)
    assert glass.medium_inside == 0
    water = s.media[0]
    np.testing.assert_allclose(water.sigma_s, np.maximum(rgb_to_spectrum((1, 1, 1)), 0))
    assert water.phase == abi.PHASE_HENYEY_GREENSTEIN and water.phase_g == 0.5
    lamp = s.materials[int(smat[1])]
    np.testing.assert_allclose(lamp.emission, rgb_to_spectrum((20, 20, 20)))
    # The OBJ cube: faces of OBJ material `grey` map to `walls`, the others to `metal`.
    v, n, t, mat = _tris(s)
    kinds = sorted(s.materials[m].shader for m in mat)
    assert kinds.count(abi.SHADER_DIFFUSE) == 6 and kinds.count(abi.SHADER_MICROFACET) == 6
    assert [e.kind for e in s.env_lights] == [abi.ENV_SUN, abi.ENV_DOME]
    d = np.array(s.env_lights[0].dir)
    np.testing.assert_allclose(d, -np.array([0.2, 1, 0.1]) / np.linalg.norm([0.2, 1, 0.1]))
    assert len(s.point_lights) == 1


def test_nff_yaml_section():
    text = ("yaml{\nshader:\n  class: glossy\n  name: shiny\n  alpha: 0.3\n  rgb: [1, 1, 1]\n  x: 0.5\n"
            "material:\n  name: shinymat\n}yaml\ns 0 0 0 1\n")
    s = parse_nff(text)
    m = s.materials[int(s.sphere_arrays()[1][0])]
    assert m.shader == abi.SHADER_MICROFACET and m.alpha == pytest.approx(0.3)
    np.testing.assert_allclose(m.reflectance, rgb_to_spectrum((0.5, 0.5, 0.5)))


REFSCENES = Path(__file__).parent / "golden" / "refscenes"


def test_collada_unit_cube():
    """unitcube.dae: 12 triangles in centimetres (<unit meter="0.01">), scaled to a unit cube
    centred at the origin; one normal per face corner, pointing outwards."""
    from naivetrace_b200.nff import load_dae
    v, n, t, names, uv = load_dae(REFSCENES / "unitcube.dae")
    assert len(t) == 12 and n is not None and uv is not None
    np.testing.assert_allclose(v.min(axis=0), [-0.5] * 3)
    np.testing.assert_allclose(v.max(axis=0), [0.5] * 3)
    tri = v[t]
    centre = tri.mean(axis=1)
    assert np.all(np.einsum("ij,ij->i", n[t[:, 0]], centre) > 0)


def test_collada_cornell_box_materials():
    """cornelbox.dae: the node translation, per face-set material symbols bound to the named
    materials of <library_materials>."""
    from naivetrace_b200.nff import load_dae
    v, n, t, names, uv = load_dae(REFSCENES / "cornelbox.dae")
    assert sorted(set(names)) == ["blue", "green", "red", "white"]
    np.testing.assert_allclose(v.min(axis=0), [-0.5, 0.0, -1.2], atol=1e-9)
    np.testing.assert_allclose(v.max(axis=0), [0.5, 1.0, 0.0], atol=1e-9)


@pytest.mark.parametrize("path", sorted(REFSCENES.glob("*.nff")), ids=lambda p: p.stem)
def test_reference_scenes_parse(path):
    s = parse_nff(path, width=16, height=16)
    assert s.num_triangles + s.num_spheres > 0
    if path.stem in ("refractive_sphere_caustics", "refract_beam_at_cube"):
        assert len(s.textures) == 1 and s.uv_array() is not None
        tex = [m for m in s.materials if m.diffuse_texture >= 0]
        assert tex and s.textures[0].shape[2] == 3 and s.textures[0].max() <= 1.0
    if path.stem == "litcorner2":
        em = [m for m in s.materials if m.emission is not None]
        assert len(em) == 1 and not em[0].emission.any()  # parallel: an emitter that radiates nothing here


def test_srgb_texture_is_linearised(tmp_path):
    from PIL import Image
    from naivetrace_b200.nff import read_texture
    Image.fromarray(np.array([[[0, 128, 255]]], np.uint8)).save(tmp_path / "t.png")
    t = read_texture(tmp_path / "t.png")
    np.testing.assert_allclose(t[0, 0], [0.0, ((128 / 255 + 0.055) / 1.055) ** 2.4, 1.0], rtol=1e-6)


def test_dense_dielectric_line():
    s = parse_nff("speculardensedielectric coat 0.2 0.4 0.6 0.05\ns 0 0 1 0.5\n")
    m = s.materials[int(s.sphere_arrays()[1][0])]
    assert m.shader == abi.SHADER_SPECULAR_DENSE_DIELECTRIC and m.specular_reflectivity == pytest.approx(0.05)
    np.testing.assert_allclose(m.reflectance, rgb_to_spectrum((0.2, 0.4, 0.6)))
