"""ctypes mirror of include/toytrace_gpu.h and the loader of the CUDA library.

The structures below must match the C declarations field for field; tests/test_abi.py
checks their sizes against the compiled library's expectations.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

NBINS = 36

TT_OK = 0
TT_ERR_CUDA = 1
TT_ERR_INVALID = 2
TT_ERR_CAPACITY = 3
TT_ERR_LOOP_CAP = 4
TT_ERR_INTERRUPTED = 5
TT_ERR_NOT_READY = 6

STATUS_NAMES = {
    TT_OK: "TT_OK",
    TT_ERR_CUDA: "TT_ERR_CUDA",
    TT_ERR_INVALID: "TT_ERR_INVALID",
    TT_ERR_CAPACITY: "TT_ERR_CAPACITY",
    TT_ERR_LOOP_CAP: "TT_ERR_LOOP_CAP",
    TT_ERR_INTERRUPTED: "TT_ERR_INTERRUPTED",
    TT_ERR_NOT_READY: "TT_ERR_NOT_READY",
}

SHADER_DIFFUSE = 0
SHADER_SPECULAR_REFLECTIVE = 1
SHADER_SPECULAR_DIELECTRIC = 2
SHADER_MICROFACET = 3
SHADER_GLOSSY_DIELECTRIC = 4
SHADER_SPECULAR_DENSE_DIELECTRIC = 5

ENV_DOME = 0
ENV_SUN = 1
ENV_MAP = 2
ENV_DIRECTIONAL = 3

CAMERA_PINHOLE = 0
CAMERA_FISHEYE = 1

ALGO_PT = 0
ALGO_PT2 = 1
SAMPLE_BOTH = 0
SAMPLE_BSDF = 1
SAMPLE_LIGHTS = 2


class Material(C.Structure):
    _fields_ = [
        ("shader", C.c_int32),
        ("reflectance", C.c_float * NBINS),
        ("alpha", C.c_float),
        ("ior_ratio", C.c_float),
        ("emissive", C.c_int32),
        ("emission", C.c_float * NBINS),
        ("medium_inside", C.c_int32),
        ("medium_outside", C.c_int32),
        ("volume_boundary", C.c_int32),
        ("diffuse_texture", C.c_int32),
        ("specular_reflectivity", C.c_float),
    ]


class Texture(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("rgb", C.POINTER(C.c_float))]


PHASE_UNIFORM = 0
PHASE_RAYLEIGH = 1
PHASE_HENYEY_GREENSTEIN = 2
MEDIUM_HOMOGENEOUS = 0
MEDIUM_ATMOSPHERE = 1


class Medium(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("priority", C.c_int32),
        ("sigma_s", C.c_float * NBINS),
        ("sigma_a", C.c_float * NBINS),
        ("phase", C.c_int32),
        ("phase_g", C.c_float),
        ("planet_center", C.c_float * 3),
        ("planet_radius", C.c_float),
        ("table_size", C.c_int32),
        ("table_h0", C.c_float),
        ("table_dh", C.c_float),
        ("sigma_t", C.POINTER(C.c_float)),
        ("sigma_s_molecules", C.POINTER(C.c_float)),
        ("sigma_s_aerosols", C.POINTER(C.c_float)),
    ]


class EnvLight(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("spectrum", C.c_float * NBINS),
        ("dir", C.c_float * 3),
        ("scalar", C.c_float),
        ("scalar2", C.c_float),
        ("tex_width", C.c_int32),
        ("tex_height", C.c_int32),
        ("tex_rgb", C.POINTER(C.c_float)),
    ]


class PointLight(C.Structure):
    _fields_ = [("spectrum", C.c_float * NBINS), ("pos", C.c_float * 3)]


class Camera(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("pos", C.c_float * 3),
        ("dir", C.c_float * 3),
        ("up", C.c_float * 3),
        ("fov_deg", C.c_float),
        ("xres", C.c_int32),
        ("yres", C.c_int32),
    ]


class SceneDesc(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_uint32),
        ("vertices", C.POINTER(C.c_float)),
        ("normals", C.POINTER(C.c_float)),
        ("num_triangles", C.c_uint32),
        ("indices", C.POINTER(C.c_uint32)),
        ("material_ids", C.POINTER(C.c_uint32)),
        ("num_materials", C.c_uint32),
        ("materials", C.POINTER(Material)),
        ("num_env_lights", C.c_uint32),
        ("env_lights", C.POINTER(EnvLight)),
        ("num_point_lights", C.c_uint32),
        ("point_lights", C.POINTER(PointLight)),
        ("num_media", C.c_uint32),
        ("media", C.POINTER(Medium)),
        ("num_spheres", C.c_uint32),
        ("spheres", C.POINTER(C.c_float)),
        ("sphere_material_ids", C.POINTER(C.c_uint32)),
        ("camera", Camera),
        ("uvs", C.POINTER(C.c_float)),
        ("num_textures", C.c_uint32),
        ("textures", C.POINTER(Texture)),
    ]


class Params(C.Structure):
    _fields_ = [
        ("max_ray_depth", C.c_int32),
        ("pt_sample_mode", C.c_int32),
        ("max_samples_per_pixel", C.c_int32),
        ("wave_paths", C.c_int32),
        ("device", C.c_int32),
        ("algo", C.c_int32),
        ("qmc", C.c_int32),
        ("sort_shading", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("paths", C.c_uint64),
        ("extension_rays", C.c_uint64),
        ("shadow_rays", C.c_uint64),
        ("extend_launches", C.c_uint64),
        ("extend_ms", C.c_double),
        ("shadow_launches", C.c_uint64),
        ("shadow_ms", C.c_double),
        ("pass_ms", C.c_double),
        ("kernel_launches", C.c_uint64),
        ("node_visits", C.c_uint64),
        ("tri_tests", C.c_uint64),
        ("shadow_node_visits", C.c_uint64),
        ("shadow_tri_tests", C.c_uint64),
        ("counted_rays", C.c_uint64),
        ("bvh_nodes", C.c_uint32),
        ("bvh_node_bytes", C.c_uint32),
        ("tri_bytes", C.c_uint32),
        ("bvh_depth", C.c_uint32),
        ("error_flags", C.c_uint64),
        ("guide_records", C.c_uint64),
        ("guide_steps", C.c_uint64),
        ("guide_loss", C.c_double),
        ("guide_train_ms", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


PKG_DIR = Path(__file__).resolve().parent
LIB_DIR = PKG_DIR / "_build"
LIB_NAME = "libtoytrace_gpu.so"

# Every symbol declared in include/toytrace_gpu.h.
EXPORTED_SYMBOLS = [
    "tt_last_wave_queue_lengths",
    "tt_abi_version",
    "tt_create",
    "tt_upload_scene",
    "tt_render_pass",
    "tt_render_pass_range",
    "tt_render_pass_noalloc",
    "tt_request_interrupt",
    "tt_request_stop",
    "tt_poll_interrupt",
    "tt_stop_requested",
    "tt_read_framebuffer",
    "tt_read_accumulators",
    "tt_generate_image",
    "tt_clear_framebuffer",
    "tt_intersect_batch",
    "tt_occluded_batch",
    "tt_intersect_batch_device",
    "tt_count_traversal",
    "tt_sample_bsdf_batch",
    "tt_eval_bsdf_batch",
    "tt_sample_phase_batch",
    "tt_eval_phase_batch",
    "tt_read_accumulators_device",
    "tt_set_profiling",
    "tt_get_stats",
    "tt_reset_stats",
    "tt_last_error",
    "tt_destroy",
    "tt_set_guiding",
    "tt_guide_num_params",
    "tt_guide_get_params",
    "tt_guide_set_params",
    "tt_guide_forward_batch",
    "tt_guide_gradient_batch",
    "tt_guide_gradient_pool_batch",
    "tt_guide_train_batch",
    "tt_guide_read_records",
    "tt_guide_features_batch",
    "tt_render_views",
    "tt_views_completion_ms",
    "tt_autotune_views",
    "tt_guide_forward_batch_tc",
    "tt_guide_tree_info",
    "tt_guide_tree_mixtures",
    "tt_guide_tree_lookup_batch",
    "tt_vmf_fit_batch",
    "tt_kdtree_build_batch",
    "tt_guide_tree_quadtree",
    "tt_quadtree_fit_batch",
    "tt_quadtree_sample_batch",
]

GUIDE_LEARNED = 0
GUIDE_TREE = 1
GUIDE_NET_TCGEN05 = 0
GUIDE_NET_MMA = 1
TREE_VMF = 0
TREE_QUADTREE = 1


class View(C.Structure):
    _fields_ = [("camera", Camera), ("spp", C.c_int32)]


TUNE_MAX = 16


class TuneResult(C.Structure):
    _fields_ = [
        ("wave_paths", C.c_int32),
        ("grid", C.c_int32),
        ("ms", C.c_double),
        ("candidates", C.c_int32),
        ("candidate_wave", C.c_int32 * TUNE_MAX),
        ("candidate_grid", C.c_int32 * TUNE_MAX),
        ("candidate_ms", C.c_double * TUNE_MAX),
        ("block", C.c_int32),
        ("bvh_width", C.c_int32),
        ("candidate_block", C.c_int32 * TUNE_MAX),
        ("candidate_width", C.c_int32 * TUNE_MAX),
    ]


class GuidingParams(C.Structure):
    _fields_ = [
        ("enabled", C.c_int32),
        ("train", C.c_int32),
        ("learning_rate", C.c_float),
        ("record_pool", C.c_int32),
        ("batch", C.c_int32),
        ("steps_per_pass", C.c_int32),
        ("max_depth", C.c_int32),
        ("seed", C.c_uint64),
        ("method", C.c_int32),
        ("tree_subdivision", C.c_int32),
        ("tree_em_iters", C.c_int32),
        ("network", C.c_int32),
        ("tree_distribution", C.c_int32),
    ]


_lib = None


class TTError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def lib_path() -> Path:
    return Path(os.environ.get("TT_GPU_LIB", LIB_DIR / LIB_NAME))


def load_library() -> C.CDLL:
    """Loads the CUDA library.  Raises if it is missing: there is no CPU fallback."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not path.exists():
        raise RuntimeError(
            f"CUDA path-tracer library not found at {path}; build it with "
            "`python -m naivetrace_b200.build` (there is no CPU fallback)"
        )
    lib = C.CDLL(str(path))
    P = C.POINTER
    vp = C.c_void_p
    sig = {
        "tt_abi_version": ([], C.c_int32),
        "tt_last_wave_queue_lengths": ([vp, P(C.c_int32), C.c_int32], C.c_int32),
        "tt_create": ([P(SceneDesc), P(Params), P(vp)], C.c_int32),
        "tt_upload_scene": ([vp], C.c_int32),
        "tt_render_pass": ([vp, C.c_int32, C.c_uint64], C.c_int32),
        "tt_render_pass_range": ([vp, C.c_int32, C.c_uint64, C.c_int32, C.c_int32], C.c_int32),
        "tt_render_pass_noalloc": ([vp, C.c_int32, C.c_uint64, C.c_int32, C.c_int32, C.c_uint64, vp, vp, vp], C.c_int32),
        "tt_request_interrupt": ([vp], C.c_int32),
        "tt_request_stop": ([vp], C.c_int32),
        "tt_poll_interrupt": ([vp], C.c_int32),
        "tt_stop_requested": ([vp], C.c_int32),
        "tt_read_framebuffer": ([vp, P(C.c_float), P(C.c_uint64)], C.c_int32),
        "tt_read_accumulators": ([vp, P(C.c_double), P(C.c_double), P(C.c_uint64), P(C.c_uint64)], C.c_int32),
        "tt_generate_image": ([vp, C.c_int32, P(C.c_uint8)], C.c_int32),
        "tt_clear_framebuffer": ([vp], C.c_int32),
        "tt_intersect_batch": ([vp, P(C.c_float), C.c_int32, P(C.c_int32), P(C.c_float), P(C.c_float), P(C.c_float)], C.c_int32),
        "tt_occluded_batch": ([vp, P(C.c_float), C.c_int32, P(C.c_uint8)], C.c_int32),
        "tt_intersect_batch_device": ([vp, vp, C.c_int32, vp, vp, vp, vp, vp], C.c_int32),
        "tt_count_traversal": ([vp, P(C.c_float), C.c_int32], C.c_int32),
        "tt_sample_bsdf_batch": ([vp, C.c_int32, P(C.c_float), P(C.c_int32), C.c_int32, C.c_uint64, P(C.c_float), P(C.c_float), P(C.c_float)], C.c_int32),
        "tt_eval_bsdf_batch": ([vp, C.c_int32, P(C.c_float), P(C.c_int32), P(C.c_float), C.c_int32, P(C.c_float), P(C.c_float)], C.c_int32),
        "tt_sample_phase_batch": ([vp, C.c_int32, P(C.c_float), P(C.c_float), P(C.c_int32), C.c_int32, C.c_uint64, P(C.c_float), P(C.c_float), P(C.c_float)], C.c_int32),
        "tt_eval_phase_batch": ([vp, C.c_int32, P(C.c_float), P(C.c_float), P(C.c_int32), P(C.c_float), C.c_int32, P(C.c_float), P(C.c_float)], C.c_int32),
        "tt_read_accumulators_device": ([vp, vp, vp, vp], C.c_int32),
        "tt_set_profiling": ([vp, C.c_int32], C.c_int32),
        "tt_get_stats": ([vp, P(Stats)], C.c_int32),
        "tt_reset_stats": ([vp], C.c_int32),
        "tt_last_error": ([vp, C.c_char_p, C.c_int32], C.c_int32),
        "tt_destroy": ([vp], None),
        "tt_set_guiding": ([vp, P(GuidingParams)], C.c_int32),
        "tt_guide_num_params": ([], C.c_int32),
        "tt_guide_get_params": ([vp, P(C.c_float), C.c_int32], C.c_int32),
        "tt_guide_set_params": ([vp, P(C.c_float), C.c_int32], C.c_int32),
        "tt_guide_forward_batch": ([vp, P(C.c_float), C.c_int32, P(C.c_float)], C.c_int32),
        "tt_guide_gradient_batch": ([vp, P(C.c_float), C.c_int32, P(C.c_float), P(C.c_float)], C.c_int32),
        "tt_guide_gradient_pool_batch": ([vp, P(C.c_float), C.c_int32, C.c_int32, C.c_uint64, P(C.c_float), P(C.c_float)], C.c_int32),
        "tt_guide_train_batch": ([vp, P(C.c_float), C.c_int32, C.c_int32, C.c_float, P(C.c_float)], C.c_int32),
        "tt_guide_read_records": ([vp, P(C.c_float), C.c_int32, P(C.c_int32)], C.c_int32),
        "tt_guide_features_batch": ([vp, P(C.c_float), C.c_int32, P(C.c_float)], C.c_int32),
        "tt_render_views": ([vp, P(View), C.c_int32, C.c_uint64, P(C.c_float)], C.c_int32),
        "tt_views_completion_ms": ([vp, P(C.c_float), C.c_int32], C.c_int32),
        "tt_autotune_views": ([vp, P(View), C.c_int32, P(TuneResult)], C.c_int32),
        "tt_guide_forward_batch_tc": ([vp, P(C.c_float), C.c_int32, P(C.c_float)], C.c_int32),
        "tt_guide_tree_info": ([vp, P(C.c_int32), P(C.c_int32), P(C.c_int32), P(C.c_int64)], C.c_int32),
        "tt_guide_tree_mixtures": ([vp, P(C.c_float), C.c_int32], C.c_int32),
        "tt_guide_tree_lookup_batch": ([vp, P(C.c_float), C.c_int32, P(C.c_int32)], C.c_int32),
        "tt_vmf_fit_batch": ([P(C.c_float), C.c_int32, P(C.c_float), P(C.c_float), C.c_int32, P(C.c_float),
                              P(C.c_float)], C.c_int32),
        "tt_kdtree_build_batch": ([P(C.c_float), C.c_int32, C.c_int32, P(C.c_int32), P(C.c_int32)], C.c_int32),
        "tt_guide_tree_quadtree": ([vp, C.c_int32, C.c_int32, P(C.c_int32), P(C.c_float), P(C.c_int32)], C.c_int32),
        "tt_quadtree_fit_batch": ([P(C.c_float), P(C.c_float), C.c_int32, P(C.c_float), P(C.c_float), C.c_int32,
                                   C.c_int32, C.c_int32, P(C.c_int32), P(C.c_float), P(C.c_float), P(C.c_int32)],
                                  C.c_int32),
        "tt_quadtree_sample_batch": ([P(C.c_int32), P(C.c_float), C.c_int32, P(C.c_float), C.c_int32, P(C.c_float),
                                      P(C.c_float), P(C.c_float)], C.c_int32),
    }
    for name, (argtypes, restype) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = restype
    _lib = lib
    return lib


def last_error(lib, ctx) -> str:
    buf = C.create_string_buffer(1024)
    lib.tt_last_error(ctx, buf, 1024)
    return buf.value.decode(errors="replace")


def check(lib, ctx, status: int, what: str) -> None:
    if status != TT_OK:
        raise TTError(status, f"{what}: {last_error(lib, ctx)}")
