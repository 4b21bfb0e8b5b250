"""ORACLE -- test infrastructure only.

ctypes binding of the CPU double-precision restatement (tt_oracle.cpp) of ToyTrace's
forward path tracer.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
may use it, as the checker; the product path never calls it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libtt_oracle.so"

_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    lib = C.CDLL(str(LIB))
    P = C.POINTER
    d = P(C.c_double)
    i32 = P(C.c_int32)
    vp = C.c_void_p
    sig = {
        "or_create": ([vp, vp], vp),
        "or_destroy": ([vp], None),
        "or_last_error": ([], C.c_char_p),
        "or_intersect": ([vp, d, C.c_int, C.c_int, i32, d, d, d], C.c_int),
        "or_occluded": ([vp, d, C.c_int, P(C.c_uint8)], C.c_int),
        "or_render": ([vp, C.c_int, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, d, d, P(C.c_uint64)], C.c_int),
        "or_sample_bsdf": ([vp, C.c_int, d, i32, C.c_int, C.c_uint64, d, d, d], C.c_int),
        "or_eval_bsdf": ([vp, C.c_int, d, i32, d, C.c_int, d, d], C.c_int),
        "or_rgb_to_spectrum": ([d, d], None),
        "or_spectrum_to_rgb": ([d, d], None),
        "or_selection_to_rgb": ([d, i32, d], None),
        "or_rgb_to_selection": ([d, i32, d], None),
        "or_reflected": ([d, d, d], None),
        "or_refracted": ([d, d, C.c_double, d], C.c_int),
        "or_half_vector": ([d, d, d], None),
        "or_half_vector_refracted": ([d, d, C.c_double, d], C.c_int),
        "or_fresnel": ([C.c_double, C.c_double], C.c_double),
        "or_pcg32_stream": ([C.c_uint64, C.c_uint64, C.c_int, P(C.c_uint32)], None),
        "or_pcg32_nextdouble_first": ([C.c_uint64, C.c_uint64], C.c_double),
        "or_uniform_int_stream": ([C.c_uint64, C.c_uint64, C.c_int, C.c_int, C.c_int, i32], C.c_int),
        "or_tables": ([d, d, d], None),
        "or_eval_env": ([vp, d, i32, d, d], C.c_int),
        "or_scene_info": ([vp, d, i32], C.c_int),
        "or_medium_walk": ([vp, d, d, C.c_double, C.c_int, i32, d, i32], C.c_int),
        "or_transmittance": ([vp, d, d, C.c_double, i32, C.c_uint64, d, d], C.c_int),
        "or_atmosphere_query": ([vp, C.c_int, d, d, d, C.c_double, i32, d], C.c_int),
        "or_medium_phase_sample": ([vp, C.c_int, d, d, i32, C.c_int, C.c_uint64, d, d, d], C.c_int),
        "or_track": ([vp, d, d, i32, C.c_int, C.c_uint64, d], C.c_int),
        "or_phase_sample": ([C.c_int, C.c_double, d, C.c_int, C.c_uint64, d, d, d], C.c_int),
        "or_sobol": ([C.c_int, C.c_int, P(C.c_uint32), d], C.c_int),
        "or_sobol_matrix": ([C.c_int, C.c_int, P(C.c_uint16), P(C.c_uint32)], None),
        "or_qmc_draws": ([C.c_int, C.c_int, C.c_uint32, C.c_int, i32, C.c_uint64, d], C.c_int),
    }
    for name, (a, r) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = a
        fn.restype = r
    _lib = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


class OracleScene:
    """CPU restatement bound to one scene (the same tt_scene_desc the GPU library takes)."""

    def __init__(self, scene, params):
        self.lib = load()
        desc, keep = scene.to_desc()
        self._keep = keep
        self.scene = scene
        self.params = params
        self.h = self.lib.or_create(C.byref(desc), C.byref(params))
        if not self.h:
            raise RuntimeError("oracle rejected scene: " + self.lib.or_last_error().decode())
        self.npix = scene.camera.xres * scene.camera.yres

    def close(self):
        if self.h:
            self.lib.or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def intersect(self, rays: np.ndarray, brute_force: bool = False):
        rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 8)
        n = len(rays)
        prim = np.zeros(n, np.int32)
        t = np.zeros(n)
        u = np.zeros(n)
        v = np.zeros(n)
        self.lib.or_intersect(self.h, _dp(rays), n, int(brute_force), _ip(prim), _dp(t), _dp(u), _dp(v))
        return prim, t, u, v

    def occluded(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 8)
        out = np.zeros(len(rays), np.uint8)
        self.lib.or_occluded(self.h, _dp(rays), len(rays), out.ctypes.data_as(C.POINTER(C.c_uint8)))
        return out.astype(bool)

    def render(self, spp: int, seed: int = 1, sample_offset: int = 0, pixel_begin: int = 0, pixel_end=None,
               nthreads: int = 0, accum=None, light_accum=None):
        """Returns (accum, light_accum, splat_count) after adding spp samples per pixel."""
        if pixel_end is None:
            pixel_end = self.npix
        accum = np.zeros(3 * self.npix) if accum is None else accum
        light = np.zeros(3 * self.npix) if light_accum is None else light_accum
        cnt = C.c_uint64(0)
        rc = self.lib.or_render(self.h, spp, seed, sample_offset, pixel_begin, pixel_end, nthreads, _dp(accum),
                                _dp(light), C.byref(cnt))
        if rc != 0:
            raise RuntimeError(self.lib.or_last_error().decode())
        return accum, light, cnt.value

    def sample_bsdf(self, material: int, wi, lambda_idx, n: int, seed: int):
        wi = np.ascontiguousarray(wi, dtype=np.float64)
        li = np.ascontiguousarray(lambda_idx, dtype=np.int32)
        d = np.zeros((n, 3))
        val = np.zeros((n, 3))
        pdf = np.zeros(n)
        self.lib.or_sample_bsdf(self.h, material, _dp(wi), _ip(li), n, seed, _dp(d), _dp(val), _dp(pdf))
        return d, val, pdf

    def eval_bsdf(self, material: int, wi, lambda_idx, dirs):
        wi = np.ascontiguousarray(wi, dtype=np.float64)
        li = np.ascontiguousarray(lambda_idx, dtype=np.int32)
        dirs = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
        n = len(dirs)
        val = np.zeros((n, 3))
        pdf = np.zeros(n)
        self.lib.or_eval_bsdf(self.h, material, _dp(wi), _ip(li), _dp(dirs), n, _dp(val), _dp(pdf))
        return val, pdf

    def eval_env(self, dir_out, lambda_idx):
        d = np.ascontiguousarray(dir_out, dtype=np.float64)
        li = np.ascontiguousarray(lambda_idx, dtype=np.int32)
        val = np.zeros(3)
        pdf = C.c_double(0)
        self.lib.or_eval_env(self.h, _dp(d), _ip(li), _dp(val), C.byref(pdf))
        return val, pdf.value

    def medium_walk(self, org, dir, tfar=1e30, max_crossings=64):
        """(initial medium, [(t, medium after crossing)]) along a ray; -1 = vacuum."""
        o = np.ascontiguousarray(org, dtype=np.float64)
        dd = np.ascontiguousarray(dir, dtype=np.float64)
        media = np.zeros(max_crossings, np.int32)
        ts = np.zeros(max_crossings)
        init = C.c_int32(0)
        n = self.lib.or_medium_walk(self.h, _dp(o), _dp(dd), tfar, max_crossings, _ip(media), _dp(ts), C.byref(init))
        return init.value, list(zip(ts[:n].tolist(), media[:n].tolist()))

    def transmittance(self, org, dir, length, lambda_idx, seed=1):
        """TransmittanceEstimate from org over length: (T per wavelength, (fwd, bwd, tr))."""
        o = np.ascontiguousarray(org, dtype=np.float64)
        dd = np.ascontiguousarray(dir, dtype=np.float64)
        li = np.ascontiguousarray(lambda_idx, dtype=np.int32)
        T = np.zeros(3)
        coeff = np.zeros(3)
        self.lib.or_transmittance(self.h, _dp(o), _dp(dd), length, _ip(li), seed, _dp(T), _dp(coeff))
        return T, coeff

    def atmosphere_query(self, medium, pos, org, dir, length, lambda_idx):
        """Dict of the atmosphere model's quantities (see or_atmosphere_query)."""
        out = np.zeros(18)
        args = [np.ascontiguousarray(a, dtype=np.float64) for a in (pos, org, dir)]
        li = np.ascontiguousarray(lambda_idx, dtype=np.int32)
        rc = self.lib.or_atmosphere_query(self.h, medium, _dp(args[0]), _dp(args[1]), _dp(args[2]), length, _ip(li),
                                          _dp(out))
        if rc != 0:
            raise ValueError("not an atmosphere medium")
        return dict(altitude=out[0], lowest=out[1:4], sigma_s=out[4:7], sigma_t=out[7:10], sigma_s_mol=out[10:13],
                    sigma_s_aer=out[13:16], segment_majorant=out[16], majorant=out[17])

    def track(self, org, dir, lambda_idx, n, seed=1):
        """n samples of the next interaction: columns interacted, distance, weight[3],
        sigma_s[3], volume pdf coefficients (forward, backward, transmittance)."""
        o = np.ascontiguousarray(org, dtype=np.float64)
        dd = np.ascontiguousarray(dir, dtype=np.float64)
        li = np.ascontiguousarray(lambda_idx, dtype=np.int32)
        out = np.zeros((n, 11))
        self.lib.or_track(self.h, _dp(o), _dp(dd), _ip(li), n, seed, _dp(out))
        return out

    def medium_phase_sample(self, medium, pos, wi, lambda_idx, n, seed=1):
        """(dirs, values per wavelength, pdf) of n phase samples at a volume vertex at pos."""
        p = np.ascontiguousarray(pos, dtype=np.float64)
        w = np.ascontiguousarray(wi, dtype=np.float64)
        li = np.ascontiguousarray(lambda_idx, dtype=np.int32)
        dirs, val, pdf = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n)
        self.lib.or_medium_phase_sample(self.h, medium, _dp(p), _dp(w), _ip(li), n, seed, _dp(dirs), _dp(val),
                                        _dp(pdf))
        return dirs, val, pdf

    def info(self):
        bb = np.zeros(6)
        cnt = np.zeros(4, np.int32)
        self.lib.or_scene_info(self.h, _dp(bb), _ip(cnt))
        return bb, cnt


def phase_sample(kind: int, g: float, wi, n: int, seed: int = 1):
    """(dirs, pdf, value) of n phase-function samples about the reverse incident direction wi."""
    lib = load()
    w = np.ascontiguousarray(wi, dtype=np.float64)
    dirs = np.zeros((n, 3))
    pdf = np.zeros(n)
    val = np.zeros(n)
    lib.or_phase_sample(kind, g, _dp(w), n, seed, _dp(dirs), _dp(pdf), _dp(val))
    return dirs, pdf, val


def combine(accum, light, samples_per_pixel, splat_count, npix):
    """Spectral3ImageBuffer::ToImage before the clamp (renderbuffer.hxx:172-200)."""
    w = npix / splat_count if splat_count > 0 else 0.0
    return accum / samples_per_pixel + w * light
