"""Python host mirror of ToyTrace's RenderingAlgo interface over the CUDA C ABI.

RenderingAlgo (src/renderingalgorithms_interface.hxx:13-30):
    SetInterruptCallback(cb)  InitializeScene(scene)  Run()  RequestInterrupt()
    RequestFullStop()  GenerateImage()
GpuPathTracer implements it with the SamplesPerPixelSchedule of the reference's
SimplePixelByPixelRenderingAlgo (renderingalgorithms_simplebase.hxx:34-157): the samples
per pass double from 1 up to 1024, capped by max_samples_per_pixel; the callback runs on
the Run thread after every pass with is_complete_pass=True; RequestInterrupt makes Run
call the callback with is_complete_pass=False at the next pass boundary; RequestFullStop
ends Run at the next wave boundary.  Both may be called from any thread, also before Run.

GpuContext is the thin object wrapper of the C ABI used by the tests and the benchmark.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Optional

import numpy as np

from . import abi
from .image import to_image
from .scene import Scene, make_params


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


class GpuContext:
    """One tt_ctx: a scene uploaded to one GPU plus its accumulators."""

    def __init__(self, scene: Scene, params: Optional[abi.Params] = None, upload: bool = True):
        self.lib = abi.load_library()
        self.scene = scene
        self.params = params if params is not None else make_params()
        desc, keep = scene.to_desc()
        self._keep = keep
        h = C.c_void_p()
        st = self.lib.tt_create(C.byref(desc), C.byref(self.params), C.byref(h))
        if st != abi.TT_OK:
            raise abi.TTError(st, "tt_create: " + abi.last_error(self.lib, None))
        self.h = h
        self.npix = scene.camera.xres * scene.camera.yres
        if upload:
            self.upload()

    def _check(self, st, what):
        abi.check(self.lib, self.h, st, what)

    def upload(self):
        self._check(self.lib.tt_upload_scene(self.h), "tt_upload_scene")

    def render_pass(self, spp: int, seed: int = 1, pixel_begin: int = 0, pixel_end: Optional[int] = None) -> int:
        if pixel_end is None and pixel_begin == 0:
            return self.lib.tt_render_pass(self.h, spp, seed)
        pe = self.npix if pixel_end is None else pixel_end
        return self.lib.tt_render_pass_range(self.h, spp, seed, pixel_begin, pe)

    def render(self, spp: int, seed: int = 1, pixel_begin: int = 0, pixel_end: Optional[int] = None) -> None:
        self._check(self.render_pass(spp, seed, pixel_begin, pixel_end), "tt_render_pass")

    def framebuffer(self) -> np.ndarray:
        rgb = np.zeros(3 * self.npix, np.float32)
        self._check(self.lib.tt_read_framebuffer(self.h, _fp(rgb), None), "tt_read_framebuffer")
        return rgb

    def accumulators(self):
        acc = np.zeros(3 * self.npix)
        light = np.zeros(3 * self.npix)
        spp = np.zeros(self.npix, np.uint64)
        splat = C.c_uint64(0)
        dp = C.POINTER(C.c_double)
        self._check(self.lib.tt_read_accumulators(self.h, acc.ctypes.data_as(dp), light.ctypes.data_as(dp),
                                                  spp.ctypes.data_as(C.POINTER(C.c_uint64)), C.byref(splat)),
                    "tt_read_accumulators")
        return acc, light, spp, splat.value

    def image(self, linear_output: bool = False) -> np.ndarray:
        out = np.zeros((self.scene.camera.yres, self.scene.camera.xres, 3), np.uint8)
        self._check(self.lib.tt_generate_image(self.h, int(linear_output), out.ctypes.data_as(C.POINTER(C.c_uint8))),
                    "tt_generate_image")
        return out

    def clear(self):
        self._check(self.lib.tt_clear_framebuffer(self.h), "tt_clear_framebuffer")

    def intersect(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = len(rays)
        prim = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        u = np.zeros(n, np.float32)
        v = np.zeros(n, np.float32)
        self._check(self.lib.tt_intersect_batch(self.h, _fp(rays), n, prim.ctypes.data_as(C.POINTER(C.c_int32)),
                                                _fp(t), _fp(u), _fp(v)), "tt_intersect_batch")
        return prim, t, u, v

    def occluded(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        out = np.zeros(len(rays), np.uint8)
        self._check(self.lib.tt_occluded_batch(self.h, _fp(rays), len(rays), out.ctypes.data_as(C.POINTER(C.c_uint8))),
                    "tt_occluded_batch")
        return out.astype(bool)

    def count_traversal(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        self._check(self.lib.tt_count_traversal(self.h, _fp(rays), len(rays)), "tt_count_traversal")

    def sample_bsdf(self, material: int, wi, lambda_idx, n: int, seed: int):
        wi = np.ascontiguousarray(wi, dtype=np.float32)
        li = np.ascontiguousarray(lambda_idx, dtype=np.int32)
        d = np.zeros((n, 3), np.float32)
        val = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        self._check(self.lib.tt_sample_bsdf_batch(self.h, material, _fp(wi), li.ctypes.data_as(C.POINTER(C.c_int32)),
                                                  n, seed, _fp(d), _fp(val), _fp(pdf)), "tt_sample_bsdf_batch")
        return d, val, pdf

    def eval_bsdf(self, material: int, wi, lambda_idx, dirs):
        wi = np.ascontiguousarray(wi, dtype=np.float32)
        li = np.ascontiguousarray(lambda_idx, dtype=np.int32)
        dirs = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1, 3)
        n = len(dirs)
        val = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        self._check(self.lib.tt_eval_bsdf_batch(self.h, material, _fp(wi), li.ctypes.data_as(C.POINTER(C.c_int32)),
                                                _fp(dirs), n, _fp(val), _fp(pdf)), "tt_eval_bsdf_batch")
        return val, pdf

    def sample_phase(self, medium: int, pos, wi, lambda_idx, n: int, seed: int):
        """(dirs, values per wavelength, pdf) of n phase-function samples of medium `medium`
        at a volume vertex at pos; wi is the reverse incident direction."""
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        wi = np.ascontiguousarray(wi, dtype=np.float32)
        li = np.ascontiguousarray(lambda_idx, dtype=np.int32)
        d = np.zeros((n, 3), np.float32)
        val = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        self._check(self.lib.tt_sample_phase_batch(self.h, medium, _fp(pos), _fp(wi),
                                                   li.ctypes.data_as(C.POINTER(C.c_int32)), n, seed, _fp(d),
                                                   _fp(val), _fp(pdf)), "tt_sample_phase_batch")
        return d, val, pdf

    def eval_phase(self, medium: int, pos, wi, lambda_idx, dirs):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        wi = np.ascontiguousarray(wi, dtype=np.float32)
        li = np.ascontiguousarray(lambda_idx, dtype=np.int32)
        dirs = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1, 3)
        n = len(dirs)
        val = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        self._check(self.lib.tt_eval_phase_batch(self.h, medium, _fp(pos), _fp(wi),
                                                 li.ctypes.data_as(C.POINTER(C.c_int32)), _fp(dirs), n, _fp(val),
                                                 _fp(pdf)), "tt_eval_phase_batch")
        return val, pdf

    def queue_lengths(self, bounces: int) -> np.ndarray:
        """(bounces, 3) extension / shadow / finished counts of the last wave."""
        out = np.zeros(3 * bounces, np.int32)
        self._check(self.lib.tt_last_wave_queue_lengths(self.h, out.ctypes.data_as(C.POINTER(C.c_int32)), bounces),
                    "tt_last_wave_queue_lengths")
        return out.reshape(bounces, 3)

    def set_profiling(self, level: int):
        self._check(self.lib.tt_set_profiling(self.h, level), "tt_set_profiling")

    def stats(self) -> dict:
        s = abi.Stats()
        self._check(self.lib.tt_get_stats(self.h, C.byref(s)), "tt_get_stats")
        return s.as_dict()

    def reset_stats(self):
        self._check(self.lib.tt_reset_stats(self.h), "tt_reset_stats")

    # Learned guiding ---------------------------------------------------------------
    def set_guiding(self, enabled: bool = True, train: int = 1, learning_rate: float = 1e-3,
                    record_pool: int = 1 << 16, batch: int = 8192, steps_per_pass: int = 16, max_depth: int = 2,
                    seed: int = 1, method: int = abi.GUIDE_LEARNED, tree_subdivision: int = 100,
                    tree_em_iters: int = 0, network: int = abi.GUIDE_NET_TCGEN05,
                    tree_distribution: int = abi.TREE_VMF):
        """train: 0 frozen, 1 collect records and train after every pass, 2 collect only;
        max_depth: guide the first max_depth bounces only (0: all).  Guiding the first two
        bounces measured the best time to a given relMSE on the gap-lit room (the network's
        cost grows with every guided vertex, its gain mostly comes from the first indirect
        ones);
        network: the inference kernel of the learned guider (GUIDE_NET_TCGEN05 or
        GUIDE_NET_MMA, same outputs); tree_distribution: the tree guider's per-cell
        distribution (TREE_VMF mixtures or TREE_QUADTREE, the reference's quadtrees)."""
        gp = abi.GuidingParams(int(enabled), int(train), learning_rate, record_pool, batch, steps_per_pass, max_depth,
                               seed, int(method), int(tree_subdivision), int(tree_em_iters), int(network),
                               int(tree_distribution))
        self._check(self.lib.tt_set_guiding(self.h, C.byref(gp)), "tt_set_guiding")

    def tree_info(self) -> dict:
        """Cells, kd-tree nodes, fitted rounds and records of the tree guider."""
        cells, nodes, rounds = C.c_int32(), C.c_int32(), C.c_int32()
        recs = C.c_int64()
        self._check(self.lib.tt_guide_tree_info(self.h, C.byref(cells), C.byref(nodes), C.byref(rounds),
                                                C.byref(recs)), "tt_guide_tree_info")
        return {"cells": cells.value, "nodes": nodes.value, "rounds": rounds.value, "records": recs.value}

    def tree_mixtures(self) -> np.ndarray:
        """(cells, 40): weights[8], means[8][3], concentrations[8] of every cell."""
        n = self.tree_info()["cells"]
        out = np.zeros((n, 40), np.float32)
        self._check(self.lib.tt_guide_tree_mixtures(self.h, _fp(out), n), "tt_guide_tree_mixtures")
        return out

    def tree_quadtree(self, cell: int, cap: int = 1 << 16):
        """A cell's quadtree: children (nodes, 4; -1 for a leaf) and sampling weights."""
        ch = np.zeros((cap, 4), np.int32)
        w = np.zeros(cap, np.float32)
        nn = C.c_int32(0)
        self._check(self.lib.tt_guide_tree_quadtree(self.h, int(cell), cap, _ip(ch), _fp(w), C.byref(nn)),
                    "tt_guide_tree_quadtree")
        return ch[: nn.value].copy(), w[: nn.value].copy()

    def tree_lookup(self, points) -> np.ndarray:
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        out = np.zeros(len(pts), np.int32)
        self._check(self.lib.tt_guide_tree_lookup_batch(self.h, _fp(pts), len(pts),
                                                        out.ctypes.data_as(C.POINTER(C.c_int32))),
                    "tt_guide_tree_lookup_batch")
        return out

    def guide_params(self) -> np.ndarray:
        n = self.lib.tt_guide_num_params()
        out = np.zeros(n, np.float32)
        self._check(self.lib.tt_guide_get_params(self.h, _fp(out), n), "tt_guide_get_params")
        return out

    def guide_set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._check(self.lib.tt_guide_set_params(self.h, _fp(p), len(p)), "tt_guide_set_params")

    def guide_forward(self, features: np.ndarray, tcgen05: bool = False) -> np.ndarray:
        """Network outputs (n x 48) of feature rows (n x 96); `tcgen05` runs the tensor-core
        kernel instead of the warp-level mma.sync one."""
        x = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, 96)
        out = np.zeros((len(x), 48), np.float32)
        name = "tt_guide_forward_batch_tc" if tcgen05 else "tt_guide_forward_batch"
        self._check(getattr(self.lib, name)(self.h, _fp(x), len(x), _fp(out)), name)
        return out

    def guide_gradient(self, records: np.ndarray):
        r = np.ascontiguousarray(records, dtype=np.float32).reshape(-1, 14)
        g = np.zeros(self.lib.tt_guide_num_params(), np.float32)
        loss = C.c_float(0.0)
        self._check(self.lib.tt_guide_gradient_batch(self.h, _fp(r), len(r), _fp(g), C.byref(loss)),
                    "tt_guide_gradient_batch")
        return float(loss.value), g

    def guide_gradient_pool(self, pool: np.ndarray, n: int, seed: int):
        """Gradient over a mini-batch of n records the device draws from `pool` by `seed`."""
        r = np.ascontiguousarray(pool, dtype=np.float32).reshape(-1, 14)
        g = np.zeros(self.lib.tt_guide_num_params(), np.float32)
        loss = C.c_float(0.0)
        self._check(self.lib.tt_guide_gradient_pool_batch(self.h, _fp(r), len(r), n, seed, _fp(g), C.byref(loss)),
                    "tt_guide_gradient_pool_batch")
        return float(loss.value), g

    def guide_train(self, records: np.ndarray, steps: int, learning_rate: float) -> float:
        r = np.ascontiguousarray(records, dtype=np.float32).reshape(-1, 14)
        loss = C.c_float(0.0)
        self._check(self.lib.tt_guide_train_batch(self.h, _fp(r), len(r), steps, learning_rate, C.byref(loss)),
                    "tt_guide_train_batch")
        return float(loss.value)

    def guide_records(self, max_records: int = 1 << 20) -> np.ndarray:
        """Collected training records (train = 2 collects without training), as (n, 14)."""
        out = np.zeros((max_records, 14), np.float32)
        n = C.c_int32(0)
        self._check(self.lib.tt_guide_read_records(self.h, _fp(out), max_records, C.byref(n)), "tt_guide_read_records")
        return out[: n.value]

    def guide_features(self, points: np.ndarray) -> np.ndarray:
        q = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 9)
        out = np.zeros((len(q), 96), np.float32)
        self._check(self.lib.tt_guide_features_batch(self.h, _fp(q), len(q), _fp(out)), "tt_guide_features_batch")
        return out

    # Multi-view batches -------------------------------------------------------------
    @staticmethod
    def _views(views):
        arr = (abi.View * len(views))()
        npix = 0
        for k, (cam, spp) in enumerate(views):
            arr[k].camera = cam.to_c()
            arr[k].spp = int(spp)
            npix += cam.xres * cam.yres
        return arr, npix

    def render_views(self, views, seed: int = 1):
        """views: [(CameraSpec, spp)].  Returns one (yres, xres, 3) linear float image per
        view (row 0 at the bottom, as framebuffer())."""
        arr, npix = self._views(views)
        rgb = np.zeros(3 * npix, np.float32)
        self._check(self.lib.tt_render_views(self.h, arr, len(views), seed, _fp(rgb)), "tt_render_views")
        out, o = [], 0
        for cam, _ in views:
            n = cam.xres * cam.yres
            out.append(rgb[3 * o:3 * (o + n)].reshape(cam.yres, cam.xres, 3))
            o += n
        return out

    def views_completion_ms(self, n: int) -> np.ndarray:
        """Completion time (ms after the batch started) of each view of the last render_views."""
        out = np.zeros(n, np.float32)
        self._check(self.lib.tt_views_completion_ms(self.h, _fp(out), n), "tt_views_completion_ms")
        return out

    def autotune_views(self, views) -> dict:
        arr, _ = self._views(views)
        r = abi.TuneResult()
        self._check(self.lib.tt_autotune_views(self.h, arr, len(views), C.byref(r)), "tt_autotune_views")
        k = min(r.candidates, abi.TUNE_MAX)
        return {"wave_paths": r.wave_paths, "grid": r.grid, "block": r.block, "bvh_width": r.bvh_width, "ms": r.ms,
                "candidates": [{"wave_paths": r.candidate_wave[i], "grid": r.candidate_grid[i],
                                "block": r.candidate_block[i], "bvh_width": r.candidate_width[i],
                                "ms": r.candidate_ms[i]} for i in range(k)]}

    def request_interrupt(self):
        self.lib.tt_request_interrupt(self.h)

    def request_stop(self):
        self.lib.tt_request_stop(self.h)

    def poll_interrupt(self) -> bool:
        return bool(self.lib.tt_poll_interrupt(self.h))

    def stop_requested(self) -> bool:
        return bool(self.lib.tt_stop_requested(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.tt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SamplesPerPixelSchedule:
    """renderingalgorithms_simplebase.hxx:34-62."""

    MAX_SPP_PER_ITERATION = 1024

    def __init__(self, max_spp: int):
        self.spp = 1
        self.total = 0
        self.max_spp = max_spp

    def update_for_next_pass(self):
        self.total += self.spp
        if self.spp < self.MAX_SPP_PER_ITERATION:
            self.spp *= 2
        if self.max_spp > 0 and self.total + self.spp > self.max_spp:
            self.spp = self.max_spp - self.total


class GpuPathTracer:
    """RenderingAlgo for the CUDA tracer (`--algo gpu`)."""

    def __init__(self, scene: Scene, params: Optional[abi.Params] = None, seed: int = 1, linear_output: bool = False):
        self.scene = scene
        self.params = params if params is not None else make_params()
        self.seed = seed
        self.linear_output = linear_output
        self._cb: Optional[Callable[[bool], None]] = None
        self.ctx = GpuContext(scene, self.params, upload=False)
        self.schedule = SamplesPerPixelSchedule(self.params.max_samples_per_pixel)
        self.last_status = abi.TT_OK

    def set_interrupt_callback(self, cb: Callable[[bool], None]):
        self._cb = cb

    def initialize_scene(self, scene: Optional[Scene] = None):
        self.ctx.upload()

    def run(self):
        self.initialize_scene()
        while not self.ctx.stop_requested() and self.schedule.spp > 0:
            st = self.ctx.render_pass(self.schedule.spp, self.seed)
            self.last_status = st
            if st == abi.TT_ERR_INTERRUPTED:
                break
            self.ctx._check(st, "tt_render_pass")
            if self.ctx.poll_interrupt() and self._cb:
                self._cb(False)
            if self._cb:
                self._cb(True)
            self.schedule.update_for_next_pass()

    def request_interrupt(self):
        self.ctx.request_interrupt()

    def request_full_stop(self):
        self.ctx.request_stop()

    def generate_image(self) -> np.ndarray:
        """8-bit RGB, row 0 at the top (framebuffer::ToImage)."""
        return self.ctx.image(self.linear_output)

    def linear_framebuffer(self) -> np.ndarray:
        return self.ctx.framebuffer()


class GpuPathTracer2(GpuPathTracer):
    """RenderingAlgo for the null-path CUDA tracer (`--algo pt2`, PathTracingAlgo2,
    renderingalgorithms_pathtracing2.cxx): the same pass schedule with params.algo set to
    ALGO_PT2."""

    def __init__(self, scene: Scene, params: Optional[abi.Params] = None, seed: int = 1, linear_output: bool = False):
        p = make_params()
        if params is not None:
            C.memmove(C.byref(p), C.byref(params), C.sizeof(p))
        p.algo = abi.ALGO_PT2
        super().__init__(scene, p, seed, linear_output)


def to_image_host(rgb, xres, yres, linear_output=False):
    return to_image(rgb, xres, yres, linear_output)


class GpuGuidedPathTracer(GpuPathTracer):
    """RenderingAlgo for the learned-guided CUDA tracer (`--algo gpug`), with the pass
    structure of the reference's guided tracer (PathTracingAlgo2::Run,
    renderingalgorithms_pathtracing_guided.cxx:1110-1211): one initial pass, then training
    sweeps of 2, 4, ... up to `guide_max_spp` one-sample passes, each starting from a cleared
    framebuffer; then guiding is frozen (no more records) and the regular samples-per-pixel
    schedule renders into a cleared framebuffer.  Training happens after every pass of a
    sweep: `steps_per_pass` Adam steps on mini-batches of the record pool."""

    def __init__(self, scene: Scene, params: Optional[abi.Params] = None, seed: int = 1, linear_output: bool = False,
                 guide_max_spp: int = 16, learning_rate: float = 1e-3, record_pool: int = 1 << 16,
                 batch: int = 8192, steps_per_pass: int = 16, max_depth: int = 2, guide_seed: int = 1):
        super().__init__(scene, params, seed, linear_output)
        self.guide_max_spp = guide_max_spp
        self.guiding = dict(learning_rate=learning_rate, record_pool=record_pool, batch=batch,
                            steps_per_pass=steps_per_pass, max_depth=max_depth, seed=guide_seed)
        self._pass_seed = seed

    def _pass(self, spp: int) -> bool:
        st = self.ctx.render_pass(spp, self._pass_seed)
        self._pass_seed += 1
        self.last_status = st
        if st == abi.TT_ERR_INTERRUPTED:
            return False
        self.ctx._check(st, "tt_render_pass")
        if self.ctx.poll_interrupt() and self._cb:
            self._cb(False)
        return True

    def run(self):
        self.initialize_scene()
        self.ctx.set_guiding(True, 1, **self.guiding)
        if not self.ctx.stop_requested():
            if not self._pass(1):
                return
            if self._cb:
                self._cb(True)
        n = 2
        while not self.ctx.stop_requested() and n <= self.guide_max_spp:
            self.ctx.clear()
            for _ in range(n):
                if self.ctx.stop_requested() or not self._pass(1):
                    return
            if self._cb:
                self._cb(True)
            n *= 2
        self.ctx.set_guiding(True, 0, **self.guiding)
        self.ctx.clear()
        while not self.ctx.stop_requested() and self.schedule.spp > 0:
            if not self._pass(self.schedule.spp):
                break
            if self._cb:
                self._cb(True)
            self.schedule.update_for_next_pass()


def vmf_fit_batch(records, mixture_in=None, fit_in=None, batch_iters: int = 0):
    """The tree guider's fit of one cell on the device: records (n, 4) = direction xyz and
    weight, in the order given; returns the 40-float mixture and the 36-float fit state."""
    lib = abi.load_library()
    r = np.ascontiguousarray(records, np.float32).reshape(-1, 4)
    mi = None if mixture_in is None else np.ascontiguousarray(mixture_in, np.float32)
    fi = None if fit_in is None else np.ascontiguousarray(fit_in, np.float32)
    mo = np.zeros(40, np.float32)
    fo = np.zeros(36, np.float32)
    st = lib.tt_vmf_fit_batch(_fp(r), len(r), None if mi is None else _fp(mi), None if fi is None else _fp(fi),
                              int(batch_iters), _fp(mo), _fp(fo))
    abi.check(lib, None, st, "tt_vmf_fit_batch")
    return mo, fo


def kdtree_build_batch(points, min_points: int = 100):
    """The tree guider's initial kd-tree over points (n, 3) (host code of the library, no
    GPU needed): returns (cell of every point, number of cells)."""
    lib = abi.load_library()
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    cells = np.zeros(len(pts), np.int32)
    nc = C.c_int32()
    st = lib.tt_kdtree_build_batch(_fp(pts), len(pts), int(min_points), cells.ctypes.data_as(C.POINTER(C.c_int32)),
                                   C.byref(nc))
    abi.check(lib, None, st, "tt_kdtree_build_batch")
    return cells, nc.value


def quadtree_fit_batch(dirs_a, weights_a, dirs_b=None, weights_b=None, stage: int = 0, cap: int = 1 << 16):
    """The tree guider's quadtree fit (host code of the library, no GPU needed): InitialFit +
    Bake on records A (unit directions (n, 3), weights), then with stage >= 1 IncrementalFit
    of records B, with stage >= 2 IterationUpdateAndBake.  Returns (children (nodes, 4),
    sampling weights, prior)."""
    lib = abi.load_library()
    da = np.ascontiguousarray(dirs_a, np.float32).reshape(-1, 3)
    wa = np.ascontiguousarray(weights_a, np.float32).reshape(-1)
    db = np.ascontiguousarray(dirs_b if dirs_b is not None else np.zeros((0, 3)), np.float32).reshape(-1, 3)
    wb = np.ascontiguousarray(weights_b if weights_b is not None else np.zeros(0), np.float32).reshape(-1)
    ch = np.zeros((cap, 4), np.int32)
    w = np.zeros(cap, np.float32)
    pr = np.zeros(cap, np.float32)
    nn = C.c_int32(0)
    st = lib.tt_quadtree_fit_batch(_fp(da), _fp(wa), len(da), _fp(db), _fp(wb), len(db), int(stage), cap, _ip(ch),
                                   _fp(w), _fp(pr), C.byref(nn))
    abi.check(lib, None, st, "tt_quadtree_fit_batch")
    n = nn.value
    return ch[:n].copy(), w[:n].copy(), pr[:n].copy()


def quadtree_sample_batch(children, weights, u):
    """The tree-guided kernel's quadtree sampler on the device with given uniforms u (n, 2):
    returns directions (n, 3), their densities and the densities evaluated at them."""
    lib = abi.load_library()
    ch = np.ascontiguousarray(children, np.int32).reshape(-1, 4)
    w = np.ascontiguousarray(weights, np.float32).reshape(-1)
    uu = np.ascontiguousarray(u, np.float32).reshape(-1, 2)
    n = len(uu)
    d = np.zeros((n, 3), np.float32)
    p = np.zeros(n, np.float32)
    e = np.zeros(n, np.float32)
    st = lib.tt_quadtree_sample_batch(_ip(ch), _fp(w), len(ch), _fp(uu), n, _fp(d), _fp(p), _fp(e))
    abi.check(lib, None, st, "tt_quadtree_sample_batch")
    return d, p, e
